/*
 * Launch shapes of the step kernels: CB threads per block and, per kernel,
 * the resident blocks per SM MB (register budget 65536 / (CB * MB)), written
 * by disco_b200/autotune.py from CUDA-event kernel times of one step of the
 * ragged64 workload (median of the instrumented steps, ms per step;
 * columns CB/MB):
 *
 *   fp64   kernel        128/6    128/8   128/10   128/12   128/16
 *          k_begin      0.9678   0.8130   0.7588   0.7670   0.9090   -> 10
 *          k_faces      1.0393   1.0384   1.0330   0.9063   0.8335   -> 16
 *          k_gradr      0.8574   0.7075   0.7853   0.7056   0.7301   -> 12
 *          k_flux_r     1.0824   0.9779   1.1559   1.1347   1.4408   -> 8
 *          k_update     1.2229   1.0291   1.1263   1.3098   2.3399   -> 8
 *          k_c2p        0.5846   0.4866   0.5028   0.5048   0.5845   -> 8
 *   mixed  kernel        128/6    128/8   128/10   128/12   128/16
 *          k_begin      0.6840   0.6841   0.6369   0.5824   0.5293   -> 16
 *          k_faces      0.8795   0.8788   0.8735   0.7607   0.6277   -> 16
 *          k_gradr      0.7046   0.5683   0.4863   0.4610   0.4324   -> 16
 *          k_flux_r     0.6769   0.6628   0.6360   0.6033   0.6996   -> 12
 *          k_update     1.1315   0.9534   0.9760   1.0558   1.6486   -> 8
 *          k_c2p        0.5651   0.4731   0.4832   0.4763   0.5304   -> 8
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
#define MB_GRAD 16
#endif
#ifndef MB_FLUX
#define MB_FLUX 12
#endif
#ifndef MB_UPDATE
#define MB_UPDATE 8
#endif
#ifndef MB_C2P
#define MB_C2P 8
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
#define MB_C2P 8
#endif
#endif
