/* libmumax2_compat.h -- drop-in C-ABI for the hot-path symbols of MuMax2's libmumax2.so.
 *
 * Same names, argument order and meaning as the reference, so the reference's cgo
 * wrappers (src/mumax/gpu/libmumax2.go, *_wrapper.go) link against libmm_b200.so
 * unchanged.  Conventions kept from the reference:
 *   - every array argument is float** of length nDevice(), one part per device;
 *   - a NULL part means "uniform mask of ones" where the reference allows it;
 *   - CUstream* is an array of nDevice() streams; launches are asynchronous;
 *   - functions return void (the reference aborts on CUDA errors, gpu_safe.h:36);
 *     here a failed launch is recorded and reported by mm_compat_last_status().
 * Each declaration cites the reference definition it replaces (path:line in mumax/2).
 */
#ifndef LIBMUMAX2_COMPAT_H
#define LIBMUMAX2_COMPAT_H

#include <cuda.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef MM_API
#if defined(_WIN32)
#define MM_API __declspec(dllexport)
#else
#define MM_API __attribute__((visibility("default")))
#endif
#endif

/* src/libmumax2/multigpu.cu:11-37 */
MM_API void setUsedGPUs(int* gpuIds, int Ngpu);
MM_API int nDevice(void);
MM_API int deviceId(int i);
/* 0 if every compat launch so far succeeded, else the first CUDA error code (sticky). */
MM_API int mm_compat_last_status(void);

/* src/libmumax2/torque.cu:59 */
MM_API void torqueAsync(float** tx, float** ty, float** tz, float** mx, float** my, float** mz, float** hx,
                        float** hy, float** hz, float** alpha_map, float alpha_mul, CUstream* stream, int Npart);
/* src/libmumax2/exchange6.cu:145 */
MM_API void exchange6Async(float** hx, float** hy, float** hz, float** mx, float** my, float** mz, float** msat,
                           float** aex, float Aex2_mu0MsatMul, int N0, int N1Part, int N2, int periodic0,
                           int periodic1, int periodic2, float cellSizeX, float cellSizeY, float cellSizeZ,
                           CUstream* streams);
/* src/libmumax2/uniaxialanisotropy.cu:90 */
MM_API void uniaxialAnisotropyAsync(float** hx, float** hy, float** hz, float** mx, float** my, float** mz,
                                    float** Ku1_map, float** MSat_map, float Ku2_Mu0Msat_mul, float** anisU_mapx,
                                    float anisU_mulx, float** anisU_mapy, float anisU_muly, float** anisU_mapz,
                                    float anisU_mulz, CUstream* stream, int Npart);
/* src/libmumax2/normalize.cu:45 */
MM_API void normalizeAsync(float** mx, float** my, float** mz, float** norm_map, CUstream* stream, int Npart);
/* src/libmumax2/add.cu:24,97,108,125,166,190,223,244,267 */
MM_API void addAsync(float** dst, float** a, float** b, CUstream* stream, int Npart);
MM_API void addMaddAsync(float** dst, float** a, float** b, float** c, float mul, CUstream* stream, int NPart);
MM_API void maddAsync(float** dst, float** a, float** b, float mulB, CUstream* stream, int Npart);
MM_API void vecMaddAsync(float** dstx, float** dsty, float** dstz, float** ax, float** ay, float** az, float** bx,
                         float** by, float** bz, float mulBx, float mulBy, float mulBz, CUstream* stream, int Npart);
MM_API void madd1Async(float** a, float** b, float mulB, CUstream* stream, int Npart);
MM_API void madd2Async(float** a, float** b, float mulB, float** c, float mulC, CUstream* stream, int Npart);
MM_API void cmaddAsync(float** dst, float a, float b, float** kern, float** src, CUstream* stream, int NComplexPart);
MM_API void linearCombination2Async(float** dst, float** a, float mulA, float** b, float mulB, CUstream* stream,
                                    int NPart);
MM_API void linearCombination3Async(float** dst, float** a, float mulA, float** b, float mulB, float** c, float mulC,
                                    CUstream* stream, int NPart);
/* src/libmumax2/mul.cu:24 */
MM_API void mulAsync(float** dst, float** a, float** b, CUstream* stream, int Npart);
/* src/libmumax2/kernelmul_micromag.cu:72 */
MM_API void kernelMulMicromag3DAsync(float** fftMx, float** fftMy, float** fftMz, float** fftKxx, float** fftKyy,
                                     float** fftKzz, float** fftKyz, float** fftKxz, float** fftKxy, CUstream* stream,
                                     int partLen3D);
/* src/libmumax2/copypad.cu:97,139,177 */
MM_API void zeroArrayAsync(float** A, int length, CUstream* streams);
MM_API void copyPad3DAsync(float** dst, int D0, int D1, int D2, float** src, int S0, int S1, int S2, int Ncomp,
                           CUstream* streams);
MM_API void copyUnPad3DAsync(float** dst, int D0, int D1, int D2, float** src, int S0, int S1, int S2, int Ncomp,
                             CUstream* streams);
/* src/libmumax2/reduce.cu:1029-1886: partial reductions, one partial per block; the
 * caller finishes them on the host (src/mumax/gpu/reductor.go:69-186) */
MM_API void partialSumAsync(float** input, float** output, int blocks, int threadsPerBlock, int N, CUstream* stream);
MM_API void partialSDotAsync(float** input1, float** input2, float** output, int blocks, int threadsPerBlock, int N,
                             CUstream* stream);
MM_API void partialMaxAsync(float** input, float** output, int blocks, int threadsPerBlock, int N, CUstream* stream);
MM_API void partialMinAsync(float** input, float** output, int blocks, int threadsPerBlock, int N, CUstream* stream);
MM_API void partialMaxAbsAsync(float** input, float** output, int blocks, int threadsPerBlock, int N,
                               CUstream* stream);
MM_API void partialMaxDiffAsync(float** a, float** b, float** output, int blocks, int threadsPerBlock, int N,
                                CUstream* stream);
MM_API void partialMaxSumAsync(float** a, float** b, float** output, int blocks, int threadsPerBlock, int N,
                               CUstream* stream);
MM_API void partialMaxNorm3SqAsync(float** x, float** y, float** z, float** output, int blocksPerGPU,
                                   int threadsPerBlockPerGPU, int NPerGPU, CUstream* streams);
MM_API void partialMaxNorm3SqDiffAsync(float** x1, float** y1, float** z1, float** x2, float** y2, float** z2,
                                       float** output, int blocksPerGPU, int threadsPerBlockPerGPU, int NPerGPU,
                                       CUstream* streams);
/* single-device variants (src/libmumax2/reduce.cu:1029,1217,1314,1411,1507,1601,1696,1791) */
MM_API void partialSumAsync1(float* d_idata, float* d_odata, int blocks, int threads, int size, CUstream stream);
MM_API void partialMaxAsync1(float* d_idata, float* d_odata, int blocks, int threads, int size, CUstream stream);
MM_API void partialMinAsync1(float* d_idata, float* d_odata, int blocks, int threads, int size, CUstream stream);
MM_API void partialMaxAbsAsync1(float* d_idata, float* d_odata, int blocks, int threads, int size, CUstream stream);
MM_API void partialMaxDiffAsync1(float* a, float* b, float* d_odata, int blocks, int threads, int size,
                                 CUstream stream);
MM_API void partialMaxSumAsync1(float* a, float* b, float* d_odata, int blocks, int threads, int size,
                                CUstream stream);
MM_API void partialMaxNorm3SqAsync1(float* x, float* y, float* z, float* d_odata, int blocks, int threads, int size,
                                    CUstream stream);
MM_API void partialMaxNorm3SqDiffAsync1(float* x1, float* y1, float* z1, float* x2, float* y2, float* z2,
                                        float* d_odata, int blocks, int threads, int size, CUstream stream);
/* src/libmumax2/temperature.cu:69 */
MM_API void temperature_scaleNoise(float** noise, float** alpha, float** temp, float alphaKB2tempMul, float** mSat,
                                   float mu0VgammaDtMSatMul, CUstream* stream, int Npart);
/* src/libmumax2/zhang-li_torque.cu:307 */
MM_API void zhangli_async(float** sttx, float** stty, float** sttz, float** mx, float** my, float** mz, float** jx,
                          float** jy, float** jz, float** msat, float** pol, float** ee, float** alpha,
                          const float jMul_x, const float jMul_y, const float jMul_z, const float pred,
                          const float eeMul, const float alphaMul, const int sx, const int sy, const int sz,
                          const float csx, const float csy, const float csz, const int pbc_x, const int pbc_y,
                          const int pbc_z, CUstream* stream);
/* src/libmumax2/slonczewski_torque.cu:120 */
MM_API void slonczewski_async(float** sttx, float** stty, float** sttz, float** mx, float** my, float** mz,
                              float** msat, float** px, float** py, float** pz, float** jx, float** jy, float** jz,
                              float** alphamsk, float** t_flmsk, float** polMsk, float** lambdaMsk,
                              float** epsilon_primeMsk, float pxMul, float pyMul, float pzMul, float jxMul,
                              float jyMul, float jzMul, float beta_prime, float pre_field, float meshSizeX,
                              float meshSizeY, float meshSizeZ, float alphaMul, float t_flMul, float lambdaMul,
                              int NPart, CUstream* stream);

#ifdef __cplusplus
}
#endif
#endif /* LIBMUMAX2_COMPAT_H */
