// fast_entries.h — registry entries of the specialised kernels: each macro
// expands to one fast::VariantA / VariantB initialiser naming the forward and
// inverse instantiations (fast_registry.h); included by the fast_*.cu tables.
#pragma once
#include "fast_registry.h"
#include "fft_fast.cuh"

#define A_ENTRY(T, DT, NY, M, RW, WY, NT, VY, VZ, MINB)                                                      \
    {0, 0, DT, NY, M, RW, WY, NT, VY, VZ, PassAShape<T, NY, M, RW, WY, NT, VY, VZ>::smem_bytes(),              \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, true, VY, VZ, MINB>,                                     \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, false, VY, VZ, MINB>,                                    \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, true, VY, VZ, MINB, 0, true>,                            \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, false, VY, VZ, MINB, 0, true>}
// Pass A with the column tiles copied ahead by cp.async (CP = 1)
#define AC_ENTRY(T, DT, NY, M, RW, WY, NT, VY, VZ, MINB)                                                     \
    {0, 0, DT, NY, M, RW, WY, NT, VY, VZ, PassAShape<T, NY, M, RW, WY, NT, VY, VZ>::smem_bytes(),              \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, true, VY, VZ, MINB, 1>,                                  \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, false, VY, VZ, MINB, 1>,                                 \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, true, VY, VZ, MINB, 1, true>,                            \
     (const void *)pass_a_fast<T, NY, M, RW, WY, NT, false, VY, VZ, MINB, 1, true>}
#define D_ENTRY(T, DT, NY, M, RW, WY, NT, K, VY, VZ, MINB)                                                   \
    {1, K, DT, NY, M, RW, WY, NT, VY, VZ, PassADsmemShape<T, NY, M, RW, WY, NT, K, VY, VZ>::smem_bytes(),        \
     (const void *)pass_a_dsmem<T, NY, M, RW, WY, NT, K, true, VY, VZ, MINB>,                                    \
     (const void *)pass_a_dsmem<T, NY, M, RW, WY, NT, K, false, VY, VZ, MINB>, nullptr, nullptr}
#define P_ENTRY(T, DT, NX, W, NT, V, MINB)                                                                    \
    {1, DT, NX, W, NT, V, (size_t)(((NX + 1) / 2 * 2) + 2 * NX * W) * sizeof(cx_t<T>),                          \
     (const void *)pass_b_pipe<T, NX, W, NT, true, V, MINB>, (const void *)pass_b_pipe<T, NX, W, NT, false, V, MINB>,  \
     (const void *)pass_b_pipe<T, NX, W, NT, true, V, MINB, true>,                                                  \
     (const void *)pass_b_pipe<T, NX, W, NT, false, V, MINB, true>}
// one tile buffer, refilled by cp.async while the last stage computes
#define Q_ENTRY(T, DT, NX, W, NT, V, MINB)                                                                    \
    {2, DT, NX, W, NT, V, (size_t)(((NX + 1) / 2 * 2) + NX * W) * sizeof(cx_t<T>),                              \
     (const void *)pass_b_pipe1<T, NX, W, NT, true, V, MINB>, (const void *)pass_b_pipe1<T, NX, W, NT, false, V, MINB>, \
     (const void *)pass_b_pipe1<T, NX, W, NT, true, V, MINB, true>,                                                 \
     (const void *)pass_b_pipe1<T, NX, W, NT, false, V, MINB, true>}
#define B_ENTRY(T, DT, NX, W, NT, V, MINB)                                                                    \
    {0, DT, NX, W, NT, V, (size_t)(NX + NX * W) * sizeof(cx_t<T>), (const void *)pass_b_fast<T, NX, W, NT, true, V, MINB>, \
     (const void *)pass_b_fast<T, NX, W, NT, false, V, MINB>,                                                       \
     (const void *)pass_b_fast<T, NX, W, NT, true, V, MINB, true>,                                                  \
     (const void *)pass_b_fast<T, NX, W, NT, false, V, MINB, true>}
