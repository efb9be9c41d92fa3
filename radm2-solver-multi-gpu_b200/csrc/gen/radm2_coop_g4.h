/* Generated by radm2-solver-multi-gpu_b200/mech/emit.py from mech/radm2_mech.json
 * (the RADM2 mechanism as encoded in the reference's mgpu.cu).  Do not edit. */
#pragma once
/* Cooperative kernel with 4 roles: species per role [17, 14, 15, 13], RHS ops per role [377, 379, 378, 377]; Jacobian slots per role [168, 168, 163, 160], ops [552, 553, 552, 552]; LU rows per role [14, 16, 13, 16], modelled makespan 5172 cycles; solve rows per role: forward [8, 11, 5, 7] backward [24, 13, 10, 12], modelled 1920 + 1344 cycles; operation words: lu 2261, lu_div 2148, fwd 448, bwd 526, bwd_div 526. */
#define RADM2_COOP_G4_NS 17  /* most species owned by one role */
