/* Generated by radm2-solver-multi-gpu_b200/mech/emit.py from mech/radm2_mech.json
 * (the RADM2 mechanism as encoded in the reference's mgpu.cu).  Do not edit. */
#pragma once
/* WRF -> KPP conversion, mgpu.cu:513-646 (dev_convert), 682-706 (convertWRFChemData).
 * Fields are field-major with i fastest: field[f][nj][nk][ni].  Species v takes
 * conv * max(src[f], 0) with src 0 = chem, 1 = rad; photolysis slot k takes ph[f] / 60. */
#define RADM2_WRF_VAR_SRC(X) X(0,0,2) X(1,0,13) X(2,0,14) X(3,0,40) X(4,0,1) X(5,0,22) X(6,1,19) X(7,0,20) X(8,0,21) X(9,0,27) X(10,0,28) X(11,0,30) X(12,0,31) X(13,0,7) X(14,0,16) X(15,0,19) X(16,0,41) X(17,0,12) X(18,1,16) X(19,0,32) X(20,0,10) X(21,0,38) X(22,0,18) X(23,0,24) X(24,0,6) X(25,0,23) X(26,0,39) X(27,0,25) X(28,0,26) X(29,0,36) X(30,0,34) X(31,1,25) X(32,0,33) X(33,0,35) X(34,1,10) X(35,1,11) X(36,1,4) X(37,1,27) X(38,1,23) X(39,0,26) X(40,1,8) X(41,0,11) X(42,0,9) X(43,1,9) X(44,1,17) X(45,0,5) X(46,0,37) X(47,0,8) X(48,1,5) X(49,1,24) X(50,0,43) X(51,1,18) X(52,0,42) X(53,0,17) X(54,0,29) X(55,1,14) X(56,1,15) X(57,0,4) X(58,0,3)
#define RADM2_WRF_JV_SRC(X) X(0,0) X(1,1) X(2,2) X(3,3) X(4,4) X(5,5) X(6,6) X(7,7) X(8,8) X(9,9) X(10,10) X(11,11) X(12,12) X(13,13) X(14,14) X(15,15) X(16,16) X(17,17) X(18,18) X(19,19) X(20,20) X(21,21) X(22,22) X(23,23) X(24,24) X(25,25) X(26,26) X(27,27)
#define RADM2_WRF_NCHEM_USED 44
#define RADM2_WRF_NRAD_USED 28
#define RADM2_WRF_NPH_USED 28
/* the reference's domain (ni, nk, nj) and interior window (i0, k0, j0, wi, wk, wj) */
#define RADM2_WRF_REF_GRID_INIT {48, 20, 48, 4, 0, 4, 39, 19, 39}
