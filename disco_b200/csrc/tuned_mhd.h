/*
 * Launch shapes of the MHD (Q = 9) instantiations of the step kernels: per kernel,
 * the resident blocks per SM MB (register budget 65536 / (CB * MB)), written
 * by disco_b200/autotune.py from CUDA-event kernel times of one step of the
 * config4_nz16 workload (median of the instrumented steps, ms per step;
 * columns CB/MB):
 *
 *   fp64   kernel        128/4    128/5    128/6    128/7    128/8   128/10   128/12
 *          k_begin      1.9414   1.9414   1.7468   1.5975   1.5166   1.5941   1.7050   -> 8
 *          k_grad       2.7288   2.3407   2.2743   2.2546   2.2262   2.2681   2.6733   -> 8
 *          k_flux       4.8046   4.2260   4.3233   4.4032   4.7350   6.6027   8.3230   -> 5
 *          k_update     2.8222   2.6586   2.6642   2.7488   2.9839   3.9034   5.9269   -> 5
 *          k_c2p        1.9937   1.5872   1.4421   1.3007   1.1989   1.2420   1.3012   -> 8
 *   mixed  kernel        128/4    128/5    128/6    128/7    128/8   128/10   128/12
 *          k_begin      1.3866   1.3862   1.3865   1.3866   1.3866   1.2227   1.1776   -> 12
 *          k_grad       1.3995   1.3988   1.4009   1.4008   1.3333   1.3728   1.2678   -> 12
 *          k_flux       2.4134   2.4135   2.1352   2.0572   1.9460   1.8873   2.2928   -> 10
 *          k_update     2.1891   2.0595   1.9458   1.8913   1.9089   2.0669   2.3853   -> 7
 *          k_c2p        1.9393   1.5485   1.3977   1.2502   1.1611   1.1900   1.2116   -> 8
 *
 * Values given with -D on the command line win.
 */
#pragma once
#ifdef DISCO_MIXED_TU
#ifndef MB_MHD_BEGIN
#define MB_MHD_BEGIN 12
#endif
#ifndef MB_MHD_GRAD
#define MB_MHD_GRAD 12
#endif
#ifndef MB_MHD_FLUX
#define MB_MHD_FLUX 10
#endif
#ifndef MB_MHD_UPDATE
#define MB_MHD_UPDATE 7
#endif
#ifndef MB_MHD_C2P
#define MB_MHD_C2P 8
#endif
#else
#ifndef MB_MHD_BEGIN
#define MB_MHD_BEGIN 8
#endif
#ifndef MB_MHD_GRAD
#define MB_MHD_GRAD 8
#endif
#ifndef MB_MHD_FLUX
#define MB_MHD_FLUX 5
#endif
#ifndef MB_MHD_UPDATE
#define MB_MHD_UPDATE 5
#endif
#ifndef MB_MHD_C2P
#define MB_MHD_C2P 8
#endif
#endif
