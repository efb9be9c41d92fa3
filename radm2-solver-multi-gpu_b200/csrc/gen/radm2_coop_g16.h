/* Generated by radm2-solver-multi-gpu_b200/mech/emit.py from mech/radm2_mech.json
 * (the RADM2 mechanism as encoded in the reference's mgpu.cu).  Do not edit. */
#pragma once
/* Cooperative kernel with 16 roles: species per role [1, 1, 1, 1, 1, 1, 4, 6, 5, 4, 6, 5, 5, 6, 6, 6], RHS ops per role [285, 146, 125, 136, 136, 122, 99, 99, 99, 98, 98, 99, 97, 95, 99, 95]; Jacobian slots per role [42, 40, 39, 43, 40, 44, 40, 41, 41, 42, 40, 41, 42, 40, 42, 42], ops [148, 149, 149, 148, 149, 149, 148, 148, 148, 149, 148, 148, 148, 148, 148, 148]; LU rows per role [4, 3, 2, 4, 3, 4, 4, 4, 4, 5, 4, 4, 3, 3, 3, 5], modelled makespan 4043 cycles; solve rows per role: forward [7, 11, 2, 4, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0] backward [14, 2, 4, 4, 2, 2, 2, 2, 2, 2, 2, 2, 3, 3, 5, 8], modelled 1912 + 1080 cycles. */
#define RADM2_COOP_G16_NS 6  /* most species owned by one role */
