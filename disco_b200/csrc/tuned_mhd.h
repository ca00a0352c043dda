/*
 * Launch shapes of the MHD (Q = 9) instantiations of the step kernels: per kernel,
 * the resident blocks per SM MB (register budget 65536 / (CB * MB)), written
 * by disco_b200/autotune.py from CUDA-event kernel times of one step of the
 * config4_nz16 workload (median of the instrumented steps, ms per step;
 * columns CB/MB):
 *
 *   fp64   kernel        128/4    128/5    128/6    128/7    128/8   128/10   128/12
 *          k_begin      2.0337   2.0335   1.8452   1.6906   1.6261   1.7644   1.8841   -> 8
 *          k_grad       2.5444   2.5455   2.4076   2.3245   2.2507   2.2590   2.5467   -> 8
 *          k_flux       6.5569   6.0407   6.5466   6.4051   7.0216   9.7142  12.0202   -> 5
 *          k_update     3.2236   3.1807   3.4487   3.7623   4.1120   5.7662   8.3289   -> 5
 *          k_c2p        1.9652   1.6211   1.4591   1.3302   1.2285   1.2634   1.3519   -> 8
 *   mixed  kernel        128/4    128/5    128/6    128/7    128/8   128/10   128/12
 *          k_begin      1.5646   1.5637   1.5639   1.5644   1.5659   1.4716   1.4673   -> 12
 *          k_grad       1.6005   1.5995   1.5976   1.5986   1.4992   1.4417   1.3659   -> 12
 *          k_flux       3.6875   3.6885   3.3207   3.0425   2.9040   3.1497   3.7171   -> 8
 *          k_update     2.7862   2.5500   2.3829   2.3982   2.5538   3.4816   4.5682   -> 6
 *          k_c2p        1.9211   1.5964   1.4324   1.3035   1.1794   1.1940   1.2627   -> 8
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
#define MB_MHD_FLUX 8
#endif
#ifndef MB_MHD_UPDATE
#define MB_MHD_UPDATE 6
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
