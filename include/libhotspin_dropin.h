/*
 * FP64 drop-in kernels exported by libhsb200.so with the exact names, argument order and
 * meaning of hotspin's CUDA library (libhotspin.h is the concatenation of
 * src/libhotspin/*.h, src/libhotspin/Makefile:35-38).  hotspin's Go layer
 * (src/hotspin-core/gpu/libhotspin.go and the wrap_*.go / *_wrapper.go files) binds these
 * through cgo unchanged; link against libhsb200.so instead of libhotspin.so.
 *
 * Conventions as in the reference: device pointers to FP64 structure-of-arrays in program
 * order, a NULL mask pointer means a uniform mask of 1 with the physical value carried by
 * the separate multiplier, `Npart` is the number of cells, the stream is a CUstream.
 * Launch failures are recorded for hsb_last_error() (the reference never checks them).
 */
#ifndef LIBHOTSPIN_DROPIN_H
#define LIBHOTSPIN_DROPIN_H

#include <cuda.h>

#ifdef __cplusplus
extern "C" {
#endif

/* replaces exchange6Async, src/libhotspin/exchange6.h:20 (kernel exchange6.cu:11-127) */
void exchange6Async(double* hx, double* hy, double* hz, double* mx, double* my, double* mz, double* msat0T0,
                    double* lex, int N0, int N1Part, int N2, int periodic0, int periodic1, int periodic2,
                    double msat0T0Mul, double lex2Mul_cellSizeX2, double lex2Mul_cellSizeY2,
                    double lex2Mul_cellSizeZ2, CUstream streams);

/* replaces uniaxialAnisotropyAsync, src/libhotspin/uniaxialanisotropy.h:20 */
void uniaxialAnisotropyAsync(double* hx, double* hy, double* hz, double* mx, double* my, double* mz,
                             double* Ku1_map, double* MSat_map, double Ku2_Mu0Msat_mul, double* anisU_mapx,
                             double anisU_mulx, double* anisU_mapy, double anisU_muly, double* anisU_mapz,
                             double anisU_mulz, CUstream stream, int Npart);

/* replaces llbar_torque_async, src/libhotspin/llbar-torque.h:20 */
void llbar_torque_async(double* tx, double* ty, double* tz, double* Mx, double* My, double* Mz, double* hx,
                        double* hy, double* hz, double* msat0T0, CUstream stream, int Npart);

/* replaces llbar_local00nc_async, src/libhotspin/llbar-local00nc.h:20 */
void llbar_local00nc_async(double* tx, double* ty, double* tz, double* hx, double* hy, double* hz,
                           double* msat0T0, double* lambda_xx, double* lambda_yy, double* lambda_zz,
                           const double lambdaMul_xx, const double lambdaMul_yy, const double lambdaMul_zz,
                           CUstream stream, int Npart);

/* replaces llbar_local02nc_async, src/libhotspin/llbar-local02nc.h:19 */
void llbar_local02nc_async(double* tx, double* ty, double* tz, double* mx, double* my, double* mz, double* hx,
                           double* hy, double* hz, double* msat0T0, double* mu_xx, double* mu_yy, double* mu_zz,
                           const double muMul_xx, const double muMul_yy, const double muMul_zz, CUstream stream,
                           int Npart);

/* replaces llbar_local02c_async, src/libhotspin/llbar-local02c.h:19 */
void llbar_local02c_async(double* tx, double* ty, double* tz, double* mx, double* my, double* mz, double* hx,
                          double* hy, double* hz, double* msat0T0, double* mu_xx, double* mu_yy, double* mu_zz,
                          const double muMul_xx, const double muMul_yy, const double muMul_zz, CUstream stream,
                          int Npart);

/* replaces long_field_async, src/libhotspin/long_field.h:20 */
void long_field_async(double* hx, double* hy, double* hz, double* mx, double* my, double* mz, double* msat0T0,
                      double* S, double* n, double* Tc, double* Ts, double msat0T0Mul, double SMul, double nMul,
                      double TcMul, double TsMul, int NPart, CUstream stream);

/* replaces brillouinAsync, src/libhotspin/brillouin.h:18 (Ridders root per cell) */
void brillouinAsync(double* msat0, double* msat0T0, double* T, double* Tc, double* S, const double msat0Mul,
                    const double msat0T0Mul, const double TcMul, const double SMul, int Npart, CUstream stream);

/* replaces kappaAsync, src/libhotspin/kappa.h:18 */
void kappaAsync(double* kappa, double* msat0, double* msat0T0, double* T, double* Tc, double* S, double* n,
                const double msat0Mul, const double msat0T0Mul, const double TcMul, const double SMul, int Npart,
                CUstream stream);

/* replaces temperature_scaleAnizNoise, src/libhotspin/temperature.h:19 */
void temperature_scaleAnizNoise(double* hx, double* hy, double* hz, double* mu_xx, double* mu_yy, double* mu_zz,
                                double* tempMask, double* msat0T0Mask, double muMul_xx, double muMul_yy,
                                double muMul_zz, double KB2tempMul_mu0VgammaDtMSatMul, CUstream stream, int Npart);

/* replaces mulAsync and tensSYMMVecMul, src/libhotspin/mul.h:19,21 */
void mulAsync(double* dst, double* a, double* b, CUstream stream, int Npart);
void tensSYMMVecMul(double* dstX, double* dstY, double* dstZ, double* srcX, double* srcY, double* srcZ,
                    double* kernXX, double* kernYY, double* kernZZ, double* kernYZ, double* kernXZ, double* kernXY,
                    const double srcMul, const int Nx, const int Ny, const int Nz, CUstream stream);

/* replaces copyPad3DAsync, copyUnPad3DAsync, zeroArrayAsync, src/libhotspin/copypad.h:28,30,33 */
void copyPad3DAsync(double* dst, int D0, int D1, int D2, double* src, int S0, int S1, int S2, int Ncomp,
                    CUstream streams);
void copyUnPad3DAsync(double* dst, int D0, int D1, int D2, double* src, int S0, int S1, int S2, int Ncomp,
                      CUstream streams);
void zeroArrayAsync(double* A, int N, CUstream streams);

/* replaces Qspat_async, src/libhotspin/Qspat.h:22 */
void Qspat_async(double* Q, double* T, double* k, const double kMul, const int sx, const int sy, const int sz,
                 const double csx, const double csy, const double csz, const int pbc_x, const int pbc_y,
                 const int pbc_z, CUstream stream);

/* replaces QinterAsync, src/libhotspin/Qinter.h:22 */
void QinterAsync(double* Qi, double* Ti, double* Tj, double* Gij, double GijMul, int Npart, CUstream stream);

/* replaces divAsync, src/libhotspin/div.h:20 */
void divAsync(double* dst, double* a, double* b, CUstream stream, int Npart);

/* replaces the add.cu family, src/libhotspin/add.h:20,24,28,32,36,40,45,49,61 */
void addAsync(double* dst, double* a, double* b, CUstream stream, int Npart);
void linearCombination2Async(double* dst, double* a, double mulA, double* b, double mulB, CUstream stream,
                             int NPart);
void linearCombination3Async(double* dst, double* a, double mulA, double* b, double mulB, double* c, double mulC,
                             CUstream stream, int NPart);
void addMaddAsync(double* dst, double* a, double* b, double* c, double mul, CUstream stream, int NPart);
void madd1Async(double* a, double* b, double mulB, CUstream stream, int Npart);
void madd2Async(double* a, double* b, double mulB, double* c, double mulC, CUstream stream, int Npart);
void maddAsync(double* dst, double* a, double* b, double mulB, CUstream stream, int Npart);
void vecMaddAsync(double* dstx, double* dsty, double* dstz, double* ax, double* ay, double* az, double* bx,
                  double* by, double* bz, double mulBx, double mulBy, double mulBz, CUstream stream, int Npart);
void cmaddAsync(double* dst, double a, double b, double* kern, double* src, CUstream stream, int NComplexPart);

/* replaces normalizeAsync, src/libhotspin/normalize.h:22 */
void normalizeAsync(double* mx, double* my, double* mz, CUstream stream, int Npart);

/* replaces dotMaskAsync, dotAsync, dotSignAsync, src/libhotspin/dot.h:21,28,31 */
void dotMaskAsync(double* dst, double* ax, double* ay, double* az, double* bx, double* by, double* bz, double axMul,
                  double ayMul, double azMul, double bxMul, double byMul, double bzMul, CUstream stream, int Npart);
void dotAsync(double* dst, double* ax, double* ay, double* az, double* bx, double* by, double* bz, CUstream stream,
              int Npart);
void dotSignAsync(double* dst, double* ax, double* ay, double* az, double* bx, double* by, double* bz, double* cx,
                  double* cy, double* cz, CUstream stream, int Npart);

/* replace the partial reductions of src/libhotspin/reduce.h:34,44,53,63,73,83,92,104,119;
 * output[b] for b < blocks holds block b's share, finished on the host
 * (gpu/reductor.go:69-203).  threadsPerBlock is accepted and ignored. */
void partialSumAsync(double* input, double* output, int blocksPerGPU, int threadsPerBlockPerGPU, int NPerGPU,
                     CUstream streams);
void partialSDotAsync(double* input1, double* input2, double* output, int blocks, int threadsPerBlock, int N,
                      CUstream stream);
void partialMaxAsync(double* input, double* output, int blocksPerGPU, int threadsPerBlockPerGPU, int NPerGPU,
                     CUstream streams);
void partialMinAsync(double* input, double* output, int blocksPerGPU, int threadsPerBlockPerGPU, int NPerGPU,
                     CUstream streams);
void partialMaxAbsAsync(double* input, double* output, int blocksPerGPU, int threadsPerBlockPerGPU, int NPerGPU,
                        CUstream streams);
void partialMaxDiffAsync(double* a, double* b, double* output, int blocksPerGPU, int threadsPerBlockPerGPU,
                         int NPerGPU, CUstream streams);
void partialMaxSumAsync(double* a, double* b, double* output, int blocksPerGPU, int threadsPerBlockPerGPU,
                        int NPerGPU, CUstream streams);
void partialMaxNorm3SqAsync(double* x, double* y, double* z, double* output, int blocksPerGPU,
                            int threadsPerBlockPerGPU, int NPerGPU, CUstream streams);
void partialMaxNorm3SqDiffAsync(double* x1, double* y1, double* z1, double* x2, double* y2, double* z2,
                                double* output, int blocksPerGPU, int threadsPerBlockPerGPU, int NPerGPU,
                                CUstream streams);


/* replaces cpAsync, src/libhotspin/Cp.h:20 (Debye phonon heat capacity, trapezoid on 61
 * intervals, low-temperature limit below T/Td = 0.01) */
void cpAsync(double* Cp, double* T, double* Td, double* n, const double TdMul, const int Npart, CUstream stream);

/* replaces tsAsync, src/libhotspin/Ts.h:18 (spin temperature from msat / Msat0T0, Ridders root) */
void tsAsync(double* Ts, double* msat, double* msat0T0, double* Tc, double* S, const double msatMul,
             const double msat0T0Mul, const double TcMul, const double SMul, int Npart, CUstream stream);

/* replaces wavgAsync, src/libhotspin/wavg.h:20 (weighted average of two temperatures) */
void wavgAsync(double* dst, double* a, double* b, double* w0, double* w1, double* R, double w0Mul, double w1Mul,
               double RMul, CUstream stream, int Npart);

/* replaces energyFlowAsync, src/libhotspin/energy_flow.h:18 */
void energyFlowAsync(double* w, double* mx, double* my, double* mz, double* Rx, double* Ry, double* Rz, double* Tc,
                     double* S, double* n, double SMul, int Npart, CUstream stream);

/* replaces llbar_nonlocal00nc_async, src/libhotspin/llbar-nonlocal00nc.h:20; the a1 + 1
 * neighbour uses the grid's own index (the reference's uses N1 for N2, the same when
 * N1 == N2) */
void llbar_nonlocal00nc_async(double* tx, double* ty, double* tz, double* hx, double* hy, double* hz,
                              double* msat0T0, double* lambda_e_xx, double* lambda_e_yy, double* lambda_e_zz,
                              const double lambda_eMul_xx, const double lambda_eMul_yy, const double lambda_eMul_zz,
                              const int sx, const int sy, const int sz, const double csx, const double csy,
                              const double csz, const int pbc_x, const int pbc_y, const int pbc_z, CUstream stream);
#ifdef __cplusplus
}
#endif
#endif
