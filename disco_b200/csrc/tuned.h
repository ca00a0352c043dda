/*
 * Launch shapes of the step kernels: CB threads per block and, per kernel,
 * the resident blocks per SM MB (register budget 65536 / (CB * MB)), written
 * by disco_b200/autotune.py from CUDA-event kernel times of one step of the
 * ragged64 workload (median of the instrumented steps, ms per step;
 * columns CB/MB):
 *
 *   fp64   kernel        128/4    128/6    128/8   128/10   128/12   128/16
 *          k_begin      0.9821   0.9820   0.8458   0.8223   0.8981   1.0168   -> 10
 *          k_faces      1.1839   1.1849   1.1836   1.1840   1.0344   0.9331   -> 16
 *          k_gradr      1.1764   0.8622   0.7015   0.7577   0.7007   0.7404   -> 12
 *          k_flux_r     1.3742   1.0753   0.9318   1.1581   1.1376   1.4398   -> 8
 *          k_update     1.8013   1.3897   1.2576   1.4172   1.6190   2.2188   -> 8
 *          k_c2p        0.5581   0.5581   0.4559   0.4311   0.4536   0.5867   -> 10
 *   mixed  kernel        128/4    128/6    128/8   128/10   128/12   128/16
 *          k_begin      0.8612   0.8613   0.8612   0.7483   0.7558   0.7423   -> 16
 *          k_faces      1.0732   1.0733   1.0722   1.0733   0.9361   0.7785   -> 16
 *          k_gradr      0.6646   0.6628   0.6052   0.5132   0.4639   0.4842   -> 12
 *          k_flux_r     0.7629   0.7630   0.6891   0.6339   0.5922   0.7117   -> 12
 *          k_update     1.6805   1.3242   1.2505   1.3088   1.5043   2.0909   -> 8
 *          k_c2p        0.5459   0.5450   0.4478   0.4190   0.4188   0.5867   -> 12
 *
 * Values given with -D on the command line win.
 */
#pragma once
#ifndef CB
#define CB 128
#endif
#ifndef FB
#define FB 128
#endif
#ifdef DISCO_MIXED_TU
#ifndef MB_BEGIN
#define MB_BEGIN 16
#endif
#ifndef MB_FACES
#define MB_FACES 16
#endif
#ifndef MB_GRAD
#define MB_GRAD 12
#endif
#ifndef MB_FLUX
#define MB_FLUX 12
#endif
#ifndef MB_UPDATE
#define MB_UPDATE 8
#endif
#ifndef MB_C2P
#define MB_C2P 12
#endif
#else
#ifndef MB_BEGIN
#define MB_BEGIN 10
#endif
#ifndef MB_FACES
#define MB_FACES 16
#endif
#ifndef MB_GRAD
#define MB_GRAD 12
#endif
#ifndef MB_FLUX
#define MB_FLUX 8
#endif
#ifndef MB_UPDATE
#define MB_UPDATE 8
#endif
#ifndef MB_C2P
#define MB_C2P 10
#endif
#endif
