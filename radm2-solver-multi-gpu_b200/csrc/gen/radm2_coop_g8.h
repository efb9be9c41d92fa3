/* Generated by radm2-solver-multi-gpu_b200/mech/emit.py from mech/radm2_mech.json
 * (the RADM2 mechanism as encoded in the reference's mgpu.cu).  Do not edit. */
#pragma once
/* Cooperative kernel with 8 roles: species per role [1, 7, 8, 6, 7, 10, 10, 10], RHS ops per role [285, 212, 211, 212, 212, 211, 209, 210]; Jacobian slots per role [84, 82, 80, 83, 84, 81, 79, 86], ops [284, 283, 283, 284, 284, 283, 282, 283]; LU rows per role [7, 7, 6, 7, 7, 8, 9, 8], modelled makespan 4194 cycles; solve rows per role: forward [8, 11, 3, 4, 2, 1, 1, 1] backward [17, 7, 8, 3, 6, 5, 8, 5], modelled 1912 + 1120 cycles; operation words: lu 2346, lu_div 2215, fwd 457, bwd 577, bwd_div 577. */
#define RADM2_COOP_G8_NS 10  /* most species owned by one role */
