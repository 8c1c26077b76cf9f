// FP64 drop-in replacements for hotspin's libhotspin kernels (same exported names,
// argument order and meaning as src/libhotspin/*.h, so hotspin's Go layer binds them
// unchanged through cgo).  Written for sm_100a: grid-stride loops over grids sized to the
// SM count, coalesced structure-of-arrays access, masks as nullable pointers
// (NULL = uniform 1, common_func.h:140-143), vacuum (Ms mask 0) gives zero torque/field.
//
// The reference launches each kernel with make1dconf/make3dconf (gpu_conf.cpp:67-120) and
// never checks the launch; these return void as well (the signature is the contract) and
// record launch failures for hsb_last_error().
#include <cuda.h>
#include <math.h>

#include "hsb_common.cuh"

#define DROPIN_THREADS 256

static inline int g1(long n) { return hsb_grid_1d(n, DROPIN_THREADS, 8); }
static inline cudaStream_t S(CUstream s) { return (cudaStream_t)s; }
static inline void check_launch(const char* who) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) hsb_set_error("%s: %s", who, cudaGetErrorString(e));
}

#define GRID_STRIDE(i, n) \
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (n); i += (long)gridDim.x * blockDim.x)

__device__ __forceinline__ double mu1(const double* m, long i) { return m ? m[i] : 1.0; }
__device__ __forceinline__ double mu0(const double* m, long i) { return m ? m[i] : 0.0; }

// ------------------------------------------------------------------ exchange6 (exchange6.cu)
__global__ void d_exchange6(double* __restrict__ hx, double* __restrict__ hy, double* __restrict__ hz,
                            const double* __restrict__ mx, const double* __restrict__ my,
                            const double* __restrict__ mz, const double* __restrict__ lexMsk, int N0,
                            int N1, int N2, int w0, int w1, int w2, double ms, double c0, double c1,
                            double c2) {
    const long n = (long)N0 * N1 * N2;
    GRID_STRIDE(I, n) {
        const int k = (int)(I % N2);
        const int j = (int)((I / N2) % N1);
        const int i = (int)(I / ((long)N1 * N2));
        const double l0 = mu1(lexMsk, I);
        const double l02 = l0 * l0;
        const double m0x = mx[I], m0y = my[I], m0z = mz[I];
        double Hx, Hy, Hz;
        // order of the reference: X (a0), then Z (a2), then Y (a1)
        {
            const long a = ((long)nb_lo(i, N0, w0) * N1 + j) * N2 + k;
            const long b = ((long)nb_hi(i, N0, w0) * N1 + j) * N2 + k;
            const double la = mu1(lexMsk, a), lb = mu1(lexMsk, b);
            const double p1 = harm0(l02, la * la), p2 = harm0(l02, lb * lb);
            Hx = c0 * ((p1 * mx[a] + p2 * mx[b]) - (p1 * m0x + p2 * m0x));
            Hy = c0 * ((p1 * my[a] + p2 * my[b]) - (p1 * m0y + p2 * m0y));
            Hz = c0 * ((p1 * mz[a] + p2 * mz[b]) - (p1 * m0z + p2 * m0z));
        }
        {
            const long a = ((long)i * N1 + j) * N2 + nb_lo(k, N2, w2);
            const long b = ((long)i * N1 + j) * N2 + nb_hi(k, N2, w2);
            const double la = mu1(lexMsk, a), lb = mu1(lexMsk, b);
            const double p1 = harm0(l02, la * la), p2 = harm0(l02, lb * lb);
            Hx += c2 * ((p1 * mx[a] + p2 * mx[b]) - (p1 * m0x + p2 * m0x));
            Hy += c2 * ((p1 * my[a] + p2 * my[b]) - (p1 * m0y + p2 * m0y));
            Hz += c2 * ((p1 * mz[a] + p2 * mz[b]) - (p1 * m0z + p2 * m0z));
        }
        {
            const long a = ((long)i * N1 + nb_lo(j, N1, w1)) * N2 + k;
            const long b = ((long)i * N1 + nb_hi(j, N1, w1)) * N2 + k;
            const double la = mu1(lexMsk, a), lb = mu1(lexMsk, b);
            const double p1 = harm0(l02, la * la), p2 = harm0(l02, lb * lb);
            Hx += c1 * ((p1 * mx[a] + p2 * mx[b]) - (p1 * m0x + p2 * m0x));
            Hy += c1 * ((p1 * my[a] + p2 * my[b]) - (p1 * m0y + p2 * m0y));
            Hz += c1 * ((p1 * mz[a] + p2 * mz[b]) - (p1 * m0z + p2 * m0z));
        }
        hx[I] = ms * Hx;
        hy[I] = ms * Hy;
        hz[I] = ms * Hz;
    }
}

// exchange6.cu:130-151.  As in the reference, the msat0T0 mask is accepted but not used:
// only its multiplier scales the field.
HSB_EXPORT void exchange6Async(double* hx, double* hy, double* hz, double* mx, double* my, double* mz,
                               double* msat0T0, double* lex, int N0, int N1Part, int N2, int periodic0,
                               int periodic1, int periodic2, double msat0T0Mul, double lex2Mul_cellSizeX2,
                               double lex2Mul_cellSizeY2, double lex2Mul_cellSizeZ2, CUstream stream) {
    (void)msat0T0;
    const long n = (long)N0 * N1Part * N2;
    d_exchange6<<<g1(n), DROPIN_THREADS, 0, S(stream)>>>(hx, hy, hz, mx, my, mz, lex, N0, N1Part, N2, periodic0,
                                                         periodic1, periodic2, msat0T0Mul, lex2Mul_cellSizeX2,
                                                         lex2Mul_cellSizeY2, lex2Mul_cellSizeZ2);
    check_launch("exchange6Async");
}

// ------------------------------------------------------------------ uniaxial anisotropy
__global__ void d_uniaxial(double* hx, double* hy, double* hz, const double* mx, const double* my,
                           const double* mz, const double* Ku, const double* Ms, double pre_mul,
                           const double* ux_m, double ux_mul, const double* uy_m, double uy_mul,
                           const double* uz_m, double uz_mul, int n) {
    GRID_STRIDE(i, n) {
        const double ms = mu1(Ms, i);
        if (ms == 0.0) {
            hx[i] = hy[i] = hz[i] = 0.0;
            continue;
        }
        const double pre = (pre_mul / ms) * mu1(Ku, i);
        const double ux = ux_mul * mu1(ux_m, i), uy = uy_mul * mu1(uy_m, i), uz = uz_mul * mu1(uz_m, i);
        const double l = sqrt(ux * ux + uy * uy + uz * uz);
        const double inv = (l != 0.0) ? 1.0 / l : 0.0;
        const double mu = mx[i] * (ux * inv) + my[i] * (uy * inv) + mz[i] * (uz * inv);
        hx[i] = pre * mu * ux;
        hy[i] = pre * mu * uy;
        hz[i] = pre * mu * uz;
    }
}

HSB_EXPORT void uniaxialAnisotropyAsync(double* hx, double* hy, double* hz, double* mx, double* my, double* mz,
                                        double* Ku1_map, double* MSat_map, double Ku2_Mu0Msat_mul,
                                        double* anisU_mapx, double anisU_mulx, double* anisU_mapy,
                                        double anisU_muly, double* anisU_mapz, double anisU_mulz,
                                        CUstream stream, int Npart) {
    d_uniaxial<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(hx, hy, hz, mx, my, mz, Ku1_map, MSat_map, Ku2_Mu0Msat_mul,
                                                            anisU_mapx, anisU_mulx, anisU_mapy, anisU_muly,
                                                            anisU_mapz, anisU_mulz, Npart);
    check_launch("uniaxialAnisotropyAsync");
}

// ------------------------------------------------------------------ LLBar terms
__global__ void d_torque(double* tx, double* ty, double* tz, const double* Mx, const double* My,
                         const double* Mz, const double* hx, const double* hy, const double* hz,
                         const double* ms0, int n) {
    GRID_STRIDE(i, n) {
        if (mu1(ms0, i) == 0.0) {
            tx[i] = ty[i] = tz[i] = 0.0;
            continue;
        }
        const double Hx = hx[i], Hy = hy[i], Hz = hz[i], mx = Mx[i], my = My[i], mz = Mz[i];
        tx[i] = -Hy * mz + Hz * my;  // cross(H, M), common_func.h:52-55
        ty[i] = -Hz * mx + Hx * mz;
        tz[i] = -Hx * my + Hy * mx;
    }
}

HSB_EXPORT void llbar_torque_async(double* tx, double* ty, double* tz, double* Mx, double* My, double* Mz,
                                   double* hx, double* hy, double* hz, double* msat0T0, CUstream stream,
                                   int Npart) {
    d_torque<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(tx, ty, tz, Mx, My, Mz, hx, hy, hz, msat0T0, Npart);
    check_launch("llbar_torque_async");
}

__global__ void d_local00nc(double* tx, double* ty, double* tz, const double* hx, const double* hy,
                            const double* hz, const double* ms0, const double* lxx, const double* lyy,
                            const double* lzz, double mxx, double myy, double mzz, int n) {
    GRID_STRIDE(i, n) {
        if (mu1(ms0, i) == 0.0) {
            tx[i] = ty[i] = tz[i] = 0.0;
            continue;
        }
        tx[i] = (lxx ? lxx[i] * mxx : mxx) * hx[i];
        ty[i] = (lyy ? lyy[i] * myy : myy) * hy[i];
        tz[i] = (lzz ? lzz[i] * mzz : mzz) * hz[i];
    }
}

HSB_EXPORT void llbar_local00nc_async(double* tx, double* ty, double* tz, double* hx, double* hy, double* hz,
                                      double* msat0T0, double* lambda_xx, double* lambda_yy, double* lambda_zz,
                                      const double lambdaMul_xx, const double lambdaMul_yy,
                                      const double lambdaMul_zz, CUstream stream, int Npart) {
    d_local00nc<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(tx, ty, tz, hx, hy, hz, msat0T0, lambda_xx, lambda_yy,
                                                             lambda_zz, lambdaMul_xx, lambdaMul_yy, lambdaMul_zz,
                                                             Npart);
    check_launch("llbar_local00nc_async");
}

// mode 0: diag(mu) (m.H) m (llbar-local02nc.cu); mode 1: (diag(mu)(m x H)) x m (llbar-local02c.cu)
__global__ void d_local02(double* tx, double* ty, double* tz, const double* mx, const double* my,
                          const double* mz, const double* hx, const double* hy, const double* hz,
                          const double* ms0, const double* uxx, const double* uyy, const double* uzz,
                          double mxx, double myy, double mzz, int n, int mode) {
    GRID_STRIDE(i, n) {
        if (mu1(ms0, i) == 0.0) {
            tx[i] = ty[i] = tz[i] = 0.0;
            continue;
        }
        const double m0 = mx[i], m1 = my[i], m2 = mz[i], H0 = hx[i], H1 = hy[i], H2 = hz[i];
        const double a = uxx ? uxx[i] * mxx : mxx, b = uyy ? uyy[i] * myy : myy, c = uzz ? uzz[i] * mzz : mzz;
        if (mode == 0) {
            const double mh = m0 * H0 + m1 * H1 + m2 * H2;
            tx[i] = a * (mh * m0);
            ty[i] = b * (mh * m1);
            tz[i] = c * (mh * m2);
        } else {
            // cross(m, H) with the reference's argument convention
            const double x0 = -m1 * H2 + m2 * H1, x1 = -m2 * H0 + m0 * H2, x2 = -m0 * H1 + m1 * H0;
            const double u0 = a * x0, u1 = b * x1, u2 = c * x2;
            tx[i] = -u1 * m2 + u2 * m1;
            ty[i] = -u2 * m0 + u0 * m2;
            tz[i] = -u0 * m1 + u1 * m0;
        }
    }
}

HSB_EXPORT void llbar_local02nc_async(double* tx, double* ty, double* tz, double* mx, double* my, double* mz,
                                      double* hx, double* hy, double* hz, double* msat0T0, double* mu_xx,
                                      double* mu_yy, double* mu_zz, const double muMul_xx, const double muMul_yy,
                                      const double muMul_zz, CUstream stream, int Npart) {
    d_local02<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(tx, ty, tz, mx, my, mz, hx, hy, hz, msat0T0, mu_xx, mu_yy,
                                                           mu_zz, muMul_xx, muMul_yy, muMul_zz, Npart, 0);
    check_launch("llbar_local02nc_async");
}

HSB_EXPORT void llbar_local02c_async(double* tx, double* ty, double* tz, double* mx, double* my, double* mz,
                                     double* hx, double* hy, double* hz, double* msat0T0, double* mu_xx,
                                     double* mu_yy, double* mu_zz, const double muMul_xx, const double muMul_yy,
                                     const double muMul_zz, CUstream stream, int Npart) {
    d_local02<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(tx, ty, tz, mx, my, mz, hx, hy, hz, msat0T0, mu_xx, mu_yy,
                                                           mu_zz, muMul_xx, muMul_yy, muMul_zz, Npart, 1);
    check_launch("llbar_local02c_async");
}

__global__ void d_normalize(double* mx, double* my, double* mz, int n) {
    GRID_STRIDE(i, n) {
        const double x = mx[i], y = my[i], z = mz[i];
        double l = sqrt(x * x + y * y + z * z);
        l = (l == 0.0) ? 0.0 : 1.0 / l;
        mx[i] = x * l;
        my[i] = y * l;
        mz[i] = z * l;
    }
}

HSB_EXPORT void normalizeAsync(double* mx, double* my, double* mz, CUstream stream, int Npart) {
    d_normalize<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(mx, my, mz, Npart);
    check_launch("normalizeAsync");
}

// ------------------------------------------------------------------ MFA (common_func.h:66-173)
#define HSB_LIN_RANGE 2.0e-1
#define HSB_INF_SPIN 1.0e5
#define HSB_ZERO 1.0e-32

__device__ double d_coth(double x) { return 1.0 / tanh(x); }

__device__ double d_Bj(double J, double x) {
    const double lpre = 1.0 / (2.0 * J), gpre = (2.0 * J + 1.0) * lpre;
    const double g2 = gpre * gpre, l2 = lpre * lpre, g4 = g2 * g2, l4 = l2 * l2, g6 = g4 * g2, l6 = l4 * l2,
                 g8 = g4 * g4, l8 = l4 * l4;
    const double lim = fmin(HSB_LIN_RANGE / gpre, HSB_LIN_RANGE / lpre);
    if (fabs(x) < lim)
        return ((g2 - l2) * x / 3.0) - ((g4 - l4) * x * x * x / 45.0) + ((g6 - l6) * x * x * x * x * x * 2.0 / 945.0) -
               ((g8 - l8) * x * x * x * x * x * x * x / 4725.0);
    return gpre * d_coth(gpre * x) - lpre * d_coth(lpre * x);
}

__device__ double d_dBjdx(double J, double x) {
    const double lpre = 1.0 / (2.0 * J), gpre = (2.0 * J + 1.0) * lpre;
    const double g2 = gpre * gpre, l2 = lpre * lpre, g4 = g2 * g2, l4 = l2 * l2, g6 = g4 * g2, l6 = l4 * l2,
                 g8 = g4 * g4, l8 = l4 * l4;
    const double lim = fmin(HSB_LIN_RANGE / gpre, HSB_LIN_RANGE / lpre);
    if (fabs(x) < lim)
        return ((g2 - l2) / 3.0) - ((g4 - l4) * x * x / 15.0) + ((g6 - l6) * x * x * x * x * 2.0 / 189.0) -
               ((g8 - l8) * x * x * x * x * x * x / 675.0);
    const double cl = d_coth(lpre * x), cg = d_coth(gpre * x);
    return (g2 - l2) + l2 * cl * cl - g2 * cg * cg;
}

__device__ double d_L(double x) {
    if (fabs(x) < HSB_LIN_RANGE)
        return (x / 3.0) - (x * x * x / 45.0) + (x * x * x * x * x * 2.0 / 945.0) - (x * x * x * x * x * x * x / 4725.0);
    return d_coth(x) - (1.0 / x);
}

__device__ double d_dLdx(double x) {
    if (fabs(x) < HSB_LIN_RANGE)
        return (1 / 3.0) - (x * x / 15.0) + (x * x * x * x * 2.0 / 189.0) - (x * x * x * x * x * x / 675.0);
    const double c = d_coth(x);
    return 1.0 - (c * c) + (1.0 / (x * x));
}

__global__ void d_long_field(double* hx, double* hy, double* hz, const double* mx, const double* my,
                             const double* mz, const double* ms0m, const double* Sm, const double* nm,
                             const double* Tcm, const double* Tsm, double ms0mul, double Smul, double nmul,
                             double Tcmul, double Tsmul, int n) {
    GRID_STRIDE(I, n) {
        const double Ms0 = ms0mul * mu1(ms0m, I), Sp = Smul * mu1(Sm, I), nn = nmul * mu1(nm, I),
                     Tc = Tcmul * mu1(Tcm, I), Ts = Tsmul * mu1(Tsm, I);
        const double x = mx[I], y = my[I], z = mz[I];
        const double a = sqrt(x * x + y * y + z * z);
        if (Ms0 == 0.0 || nn == 0.0 || a <= HSB_ZERO) {
            hx[I] = hy[I] = hz[I] = 0.0;
            continue;
        }
        const double inv = 1.0 / a;
        const double preS = (Sp > HSB_INF_SPIN) ? 1.0 : Sp / (Sp + 1.0);
        const double b = 3.0 * preS * Tc / Ts;
        const double meb = a * b;
        const double W = (Sp > HSB_INF_SPIN) ? d_L(meb) : d_Bj(Sp, meb);
        const double dW = (Sp > HSB_INF_SPIN) ? d_dLdx(meb) : d_dBjdx(Sp, meb);
        const double mult = nn * 1.38064881313131313E-23 * Ts * (W - a) / (4.0e-7 * M_PI * Ms0 * dW);
        hx[I] = mult * (x * inv);
        hy[I] = mult * (y * inv);
        hz[I] = mult * (z * inv);
    }
}

HSB_EXPORT void long_field_async(double* hx, double* hy, double* hz, double* mx, double* my, double* mz,
                                 double* msat0T0, double* S_, double* n, double* Tc, double* Ts, double msat0T0Mul,
                                 double SMul, double nMul, double TcMul, double TsMul, int NPart, CUstream stream) {
    d_long_field<<<g1(NPart), DROPIN_THREADS, 0, S(stream)>>>(hx, hy, hz, mx, my, mz, msat0T0, S_, n, Tc, Ts,
                                                              msat0T0Mul, SMul, nMul, TcMul, TsMul, NPart);
    check_launch("long_field_async");
}

// The self-consistency model of brillouinKern: f(n) = W(pre n) - n.
__device__ double d_model(double nn, double J, double pre) {
    const double x = pre * nn;
    return ((J > HSB_INF_SPIN) ? d_L(x) : d_Bj(J, x)) - nn;
}

__device__ double d_sign(double x) {
    const double v = (signbit(x) == 0) ? 1.0 : -1.0;
    return (x == 0.0) ? 0.0 : v;
}

// Ridders bracketing root search of findroot_Ridders (brillouin.cu:13-71) on any model f:
// the same midpoint / exponential-correction update, bracket bookkeeping, 1e10 seeds, the
// relative-change stop at 1e-8 and the 1000-iteration cap, so the roots (m_e(T) here, the spin
// temperature in tsAsync) equal the reference's to the last bit where the models agree.
template <typename F>
__device__ double d_ridders(const F& f, double xa, double xb) {
    const double ya = f(xa);
    if (fabs(ya) < HSB_ZERO) return xa;
    const double yb = f(xb);
    if (fabs(yb) < HSB_ZERO) return xb;
    double y1 = ya, x1 = xa, y2 = yb, x2 = xb;
    double x = 1.0e10, tx = x, teps = x;
    int iter = 0;
    while (teps > 1.0e-8 && iter < 1000) {
        const double x3 = 0.5 * (x2 + x1);
        const double y3 = f(x3);
        const double dy = (y3 * y3 - y1 * y2);
        if (dy == 0.0) {
            x = x3;
            break;
        }
        const double dx = (x3 - x1) * d_sign(y1 - y2) * y3 / (sqrt(dy));
        x = x3 + dx;
        const double y = f(x);
        const bool s3 = signbit(y) == signbit(y3);
        y2 = s3 ? y2 : y3;
        x2 = s3 ? x2 : x3;
        const bool s1 = (signbit(y) == signbit(y1)) || x2 == x3;
        y2 = s1 ? y2 : y1;
        x2 = s1 ? x2 : x1;
        y1 = y;
        x1 = x;
        teps = fabs((x - tx) / (tx + x));
        tx = x;
        iter++;
    }
    return x;
}

__global__ void d_brillouin(double* msat0, const double* ms0T0m, const double* T, const double* Tcm,
                            const double* Sm, double msat0Mul, double ms0T0Mul, double TcMul, double SMul, int n) {
    GRID_STRIDE(i, n) {
        const double Temp = T[i];
        const double ms0T0 = ms0T0Mul * mu1(ms0T0m, i);
        if (ms0T0 == 0.0) { msat0[i] = 0.0; continue; }
        if (Temp == 0.0) { msat0[i] = ms0T0 / msat0Mul; continue; }
        const double Tc = TcMul * mu1(Tcm, i);
        if (Temp > Tc) { msat0[i] = 0.0; continue; }
        const double Sp = SMul * mu1(Sm, i);
        const double preS = (Sp > HSB_INF_SPIN) ? 1.0 : Sp / (Sp + 1.0);
        const double pre = 3.0 * preS * (Tc / Temp);
        const double dT = (Tc - Temp) / Tc;
        const double lo = (dT < 0.0004) ? -0.1 : 0.01;
        const double hi = (dT < 0.0004) ? 0.5 : 1.1;
        const double me = d_ridders([&](double nn) { return d_model(nn, Sp, pre); }, lo, hi);
        msat0[i] = ms0T0 * fabs(me) / msat0Mul;
    }
}

HSB_EXPORT void brillouinAsync(double* msat0, double* msat0T0, double* T, double* Tc, double* S_, const double msat0Mul,
                               const double msat0T0Mul, const double TcMul, const double SMul, int Npart,
                               CUstream stream) {
    d_brillouin<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(msat0, msat0T0, T, Tc, S_, msat0Mul, msat0T0Mul, TcMul,
                                                             SMul, Npart);
    check_launch("brillouinAsync");
}

__global__ void d_kappa(double* kappa, const double* ms0m, const double* ms0T0m, const double* T, const double* Tcm,
                        const double* Sm, const double* nm, double msat0Mul, double ms0T0Mul, double TcMul,
                        double SMul, int n) {
    GRID_STRIDE(i, n) {
        const double u = mu1(ms0T0m, i);
        const double ms0T0 = ms0T0Mul * u;
        const double Temp = T[i];
        if (ms0T0 == 0.0 || Temp == 0.0) { kappa[i] = 0.0; continue; }
        const double Sp = SMul * mu1(Sm, i), Tc = TcMul * mu1(Tcm, i), msat0 = msat0Mul * mu1(ms0m, i);
        const double preS = (Sp > HSB_INF_SPIN) ? 1.0 : Sp / (Sp + 1.0);
        const double J0 = 3.0 * Tc;
        const double nn = nm ? nm[i] : 1.0;
        const double mul = u * u / (preS * J0 * nn);
        const double me = msat0 / ms0T0;
        const double b = preS * J0 / Temp;
        double f = (Sp > HSB_INF_SPIN) ? d_dLdx(me * b) : d_dBjdx(Sp, me * b);
        f = b * f;
        kappa[i] = mul * (f / (1.0 - f));
    }
}

HSB_EXPORT void kappaAsync(double* kappa, double* msat0, double* msat0T0, double* T, double* Tc, double* S_, double* n,
                           const double msat0Mul, const double msat0T0Mul, const double TcMul, const double SMul,
                           int Npart, CUstream stream) {
    d_kappa<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(kappa, msat0, msat0T0, T, Tc, S_, n, msat0Mul, msat0T0Mul,
                                                         TcMul, SMul, Npart);
    check_launch("kappaAsync");
}

// ------------------------------------------------------------------ thermal scaling (temperature.cu)
__global__ void d_scale_noise(double* hx, double* hy, double* hz, const double* uxx, const double* uyy,
                              const double* uzz, const double* Tm, const double* ms0m, double mxx, double myy,
                              double mzz, double pre_mul, int n) {
    GRID_STRIDE(i, n) {
        const double ms = mu1(ms0m, i);
        if (ms == 0.0) { hx[i] = hy[i] = hz[i] = 0.0; continue; }
        const double a = sqrt(mxx * mu1(uxx, i)), b = sqrt(myy * mu1(uyy, i)), c = sqrt(mzz * mu1(uzz, i));
        const double pre = sqrt((mu1(Tm, i) * pre_mul) / ms);
        hx[i] = pre * (a * hx[i]);
        hy[i] = pre * (b * hy[i]);
        hz[i] = pre * (c * hz[i]);
    }
}

HSB_EXPORT void temperature_scaleAnizNoise(double* hx, double* hy, double* hz, double* mu_xx, double* mu_yy,
                                           double* mu_zz, double* tempMask, double* msat0T0Mask, double muMul_xx,
                                           double muMul_yy, double muMul_zz, double KB2tempMul_mu0VgammaDtMSatMul,
                                           CUstream stream, int Npart) {
    d_scale_noise<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(hx, hy, hz, mu_xx, mu_yy, mu_zz, tempMask, msat0T0Mask,
                                                               muMul_xx, muMul_yy, muMul_zz,
                                                               KB2tempMul_mu0VgammaDtMSatMul, Npart);
    check_launch("temperature_scaleAnizNoise");
}

// ------------------------------------------------------------------ spectral multiply (mul.cu)
__global__ void d_mul(double* dst, const double* a, const double* b, int n) {
    GRID_STRIDE(i, n) dst[i] = a[i] * b[i];
}

HSB_EXPORT void mulAsync(double* dst, double* a, double* b, CUstream stream, int Npart) {
    d_mul<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dst, a, b, Npart);
    check_launch("mulAsync");
}

__global__ void d_tens_symm(double* dX, double* dY, double* dZ, const double* sX, const double* sY,
                            const double* sZ, const double* kXX, const double* kYY, const double* kZZ,
                            const double* kYZ, const double* kXZ, const double* kXY, double srcMul, int Nx,
                            int Ny, int Nz) {
    const long n = (long)Nx * Ny * Nz;
    GRID_STRIDE(I, n) {
        const int k = (int)(I % Nz);
        const int j = (int)((I / Nz) % Ny);
        const int i = (int)(I / ((long)Ny * Nz));
        const long e = 2 * I;
        const double RMX = srcMul * sX[e], IMX = srcMul * sX[e + 1];
        const double RMY = srcMul * sY[e], IMY = srcMul * sY[e + 1];
        const double RMZ = srcMul * sZ[e], IMZ = srcMul * sZ[e + 1];
        double sXY = 1.0, sXZ = 1.0, sYZ = 1.0;
        if (j > Ny / 2) { sXY = -sXY; sYZ = -sYZ; }
        const int jj = (j > Ny / 2) ? Ny - j : j;
        if (i > Nx / 2) { sXY = -sXY; sXZ = -sXZ; }
        const int ii = (i > Nx / 2) ? Nx - i : i;
        const long K = ((long)ii * (Ny / 2 + 1) + jj) * Nz + k;
        const double KXX = mu0(kXX, K), KXZ = sXZ * mu0(kXZ, K), KXY = sXY * mu0(kXY, K);
        const double KYZ = sYZ * mu0(kYZ, K), KYY = mu0(kYY, K), KZZ = mu0(kZZ, K);
        dX[e] = KXX * RMX + KXY * RMY + KXZ * RMZ;
        dX[e + 1] = KXX * IMX + KXY * IMY + KXZ * IMZ;
        dY[e] = KXY * RMX + KYY * RMY + KYZ * RMZ;
        dY[e + 1] = KXY * IMX + KYY * IMY + KYZ * IMZ;
        dZ[e] = KXZ * RMX + KYZ * RMY + KZZ * RMZ;
        dZ[e + 1] = KXZ * IMX + KYZ * IMY + KZZ * IMZ;
    }
}

// mul.cu:92-118 (in place is allowed: every element is read before it is written by the
// same thread)
HSB_EXPORT void tensSYMMVecMul(double* dstX, double* dstY, double* dstZ, double* srcX, double* srcY, double* srcZ,
                               double* kernXX, double* kernYY, double* kernZZ, double* kernYZ, double* kernXZ,
                               double* kernXY, const double srcMul, const int Nx, const int Ny, const int Nz,
                               CUstream stream) {
    const long n = (long)Nx * Ny * Nz;
    d_tens_symm<<<g1(n), DROPIN_THREADS, 0, S(stream)>>>(dstX, dstY, dstZ, srcX, srcY, srcZ, kernXX, kernYY, kernZZ,
                                                         kernYZ, kernXZ, kernXY, srcMul, Nx, Ny, Nz);
    check_launch("tensSYMMVecMul");
}

// ------------------------------------------------------------------ pad / unpad (copypad.cu)
__global__ void d_copy3d(double* dst, int D1, int D2, const double* src, int S1, int S2, int R0, int R1, int R2) {
    const long n = (long)R0 * R1 * R2;
    GRID_STRIDE(I, n) {
        const int k = (int)(I % R2);
        const int j = (int)((I / R2) % R1);
        const int i = (int)(I / ((long)R1 * R2));
        dst[((long)i * D1 + j) * D2 + k] = src[((long)i * S1 + j) * S2 + k];
    }
}

// copypad.cu:34-47: copies the S block into D (which the caller zeroed); per component.
HSB_EXPORT void copyPad3DAsync(double* dst, int D0, int D1, int D2, double* src, int S0, int S1, int S2, int Ncomp,
                               CUstream stream) {
    for (int c = 0; c < Ncomp; c++)
        d_copy3d<<<g1((long)S0 * S1 * S2), DROPIN_THREADS, 0, S(stream)>>>(
            dst + (long)c * D0 * D1 * D2, D1, D2, src + (long)c * S0 * S1 * S2, S1, S2, S0, S1, S2);
    check_launch("copyPad3DAsync");
}

// copypad.cu:83-103: crops the D block out of S; per component.
HSB_EXPORT void copyUnPad3DAsync(double* dst, int D0, int D1, int D2, double* src, int S0, int S1, int S2, int Ncomp,
                                 CUstream stream) {
    for (int c = 0; c < Ncomp; c++)
        d_copy3d<<<g1((long)D0 * D1 * D2), DROPIN_THREADS, 0, S(stream)>>>(
            dst + (long)c * D0 * D1 * D2, D1, D2, src + (long)c * S0 * S1 * S2, S1, S2, D0, D1, D2);
    check_launch("copyUnPad3DAsync");
}

__global__ void d_zero(double* a, int n) {
    GRID_STRIDE(i, n) a[i] = 0.0;
}

HSB_EXPORT void zeroArrayAsync(double* A, int length, CUstream stream) {
    d_zero<<<g1(length), DROPIN_THREADS, 0, S(stream)>>>(A, length);
    check_launch("zeroArrayAsync");
}

// ------------------------------------------------------------------ heat baths
__global__ void d_qspat(double* Q, const double* T, const double* km, double kMul, int sx, int sy, int sz,
                        double cx, double cy, double cz, int px, int py, int pz) {
    const long n = (long)sx * sy * sz;
    GRID_STRIDE(I, n) {
        const int k = (int)(I % sz);
        const int j = (int)((I / sz) % sy);
        const int i = (int)(I / ((long)sy * sz));
        const double T0 = T[I], k0 = mu1(km, I);
        double ddT;
        {
            const long a = ((long)nb_lo(i, sx, px) * sy + j) * sz + k, b = ((long)nb_hi(i, sx, px) * sy + j) * sz + k;
            const double p1 = harm0(k0, mu1(km, a)), p2 = harm0(k0, mu1(km, b));
            ddT = cx * ((p1 * T[a] + p2 * T[b]) - (p1 * T0 + p2 * T0));
        }
        {
            const long a = ((long)i * sy + j) * sz + nb_lo(k, sz, pz), b = ((long)i * sy + j) * sz + nb_hi(k, sz, pz);
            const double p1 = harm0(k0, mu1(km, a)), p2 = harm0(k0, mu1(km, b));
            ddT += cz * ((p1 * T[a] + p2 * T[b]) - (p1 * T0 + p2 * T0));
        }
        {
            const long a = ((long)i * sy + nb_lo(j, sy, py)) * sz + k, b = ((long)i * sy + nb_hi(j, sy, py)) * sz + k;
            const double p1 = harm0(k0, mu1(km, a)), p2 = harm0(k0, mu1(km, b));
            ddT += cy * ((p1 * T[a] + p2 * T[b]) - (p1 * T0 + p2 * T0));
        }
        Q[I] = kMul * ddT;
    }
}

HSB_EXPORT void Qspat_async(double* Q, double* T, double* k, const double kMul, const int sx, const int sy,
                            const int sz, const double csx, const double csy, const double csz, const int pbc_x,
                            const int pbc_y, const int pbc_z, CUstream stream) {
    const long n = (long)sx * sy * sz;
    d_qspat<<<g1(n), DROPIN_THREADS, 0, S(stream)>>>(Q, T, k, kMul, sx, sy, sz, 1.0 / (csx * csx), 1.0 / (csy * csy),
                                                     1.0 / (csz * csz), pbc_x, pbc_y, pbc_z);
    check_launch("Qspat_async");
}

__global__ void d_qinter(double* Qi, const double* Ti, const double* Tj, const double* G, double GMul, int n) {
    GRID_STRIDE(i, n) Qi[i] = (G ? GMul * G[i] : GMul) * (Tj[i] - Ti[i]);
}

HSB_EXPORT void QinterAsync(double* Qi, double* Ti, double* Tj, double* Gij, double GijMul, int Npart,
                            CUstream stream) {
    d_qinter<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(Qi, Ti, Tj, Gij, GijMul, Npart);
    check_launch("QinterAsync");
}

__global__ void d_div(double* dst, const double* a, const double* b, int n) {
    GRID_STRIDE(i, n) {
        const double bb = b ? b[i] : 1.0;
        dst[i] = (bb == 0.0) ? 0.0 : a[i] / bb;
    }
}

HSB_EXPORT void divAsync(double* dst, double* a, double* b, CUstream stream, int Npart) {
    d_div<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dst, a, b, Npart);
    check_launch("divAsync");
}

// ------------------------------------------------------------------ linear algebra (add.cu)
// dst = ca*a + cb*b + cc*c (+ cs) with nullable operands; one kernel covers the add.cu family.
__global__ void d_lincomb(double* dst, const double* a, double ca, const double* b, double cb, const double* c,
                          double cc, double cs, int bnull_is_one, int n) {
    GRID_STRIDE(i, n) {
        double v = cs;
        if (a) v += ca * a[i];
        if (b) v += cb * b[i];
        else if (bnull_is_one) v += cb;
        if (c) v += cc * c[i];
        dst[i] = v;
    }
}

HSB_EXPORT void addAsync(double* dst, double* a, double* b, CUstream stream, int Npart) {
    d_lincomb<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dst, a, 1.0, b, 1.0, nullptr, 0.0, 0.0, 0, Npart);
    check_launch("addAsync");
}

__global__ void d_addmadd(double* dst, const double* a, const double* b, const double* c, double mul, int n) {
    GRID_STRIDE(i, n) dst[i] = a[i] + mul * (b[i] + c[i]);
}

HSB_EXPORT void addMaddAsync(double* dst, double* a, double* b, double* c, double mul, CUstream stream, int NPart) {
    d_addmadd<<<g1(NPart), DROPIN_THREADS, 0, S(stream)>>>(dst, a, b, c, mul, NPart);
    check_launch("addMaddAsync");
}

// add.cu:95-108: b == NULL adds the scalar mulB
HSB_EXPORT void maddAsync(double* dst, double* a, double* b, double mulB, CUstream stream, int Npart) {
    d_lincomb<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dst, a, 1.0, b, mulB, nullptr, 0.0, 0.0, 1, Npart);
    check_launch("maddAsync");
}

HSB_EXPORT void vecMaddAsync(double* dstx, double* dsty, double* dstz, double* ax, double* ay, double* az, double* bx,
                             double* by, double* bz, double mulBx, double mulBy, double mulBz, CUstream stream,
                             int Npart) {
    d_lincomb<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dstx, ax, 1.0, bx, mulBx, nullptr, 0.0, 0.0, 1, Npart);
    d_lincomb<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dsty, ay, 1.0, bx ? by : nullptr, mulBy, nullptr, 0.0, 0.0, 1,
                                                           Npart);
    d_lincomb<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dstz, az, 1.0, bx ? bz : nullptr, mulBz, nullptr, 0.0, 0.0, 1,
                                                           Npart);
    check_launch("vecMaddAsync");
}

// add.cu:137-150: a += mulB * (b or 1)
HSB_EXPORT void madd1Async(double* a, double* b, double mulB, CUstream stream, int Npart) {
    d_lincomb<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(a, a, 1.0, b, mulB, nullptr, 0.0, 0.0, 1, Npart);
    check_launch("madd1Async");
}

__global__ void d_madd2(double* a, const double* b, double mulB, const double* c, double mulC, int n) {
    GRID_STRIDE(i, n) {
        const double B = b ? b[i] : 1.0, C = c ? c[i] : 1.0;
        a[i] += mulB * B + mulC * C;
    }
}

HSB_EXPORT void madd2Async(double* a, double* b, double mulB, double* c, double mulC, CUstream stream, int Npart) {
    d_madd2<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(a, b, mulB, c, mulC, Npart);
    check_launch("madd2Async");
}

__global__ void d_cmadd(double* dst, double a, double b, const double* kern, const double* src, int n) {
    GRID_STRIDE(i, n) {
        const long e = 2 * i;
        const double Sa = src[e], Sb = src[e + 1], k = kern[i];
        dst[e] += k * (a * Sa - b * Sb);
        dst[e + 1] += k * (b * Sa + a * Sb);
    }
}

HSB_EXPORT void cmaddAsync(double* dst, double a, double b, double* kern, double* src, CUstream stream,
                           int NComplexPart) {
    d_cmadd<<<g1(NComplexPart), DROPIN_THREADS, 0, S(stream)>>>(dst, a, b, kern, src, NComplexPart);
    check_launch("cmaddAsync");
}

HSB_EXPORT void linearCombination2Async(double* dst, double* a, double mulA, double* b, double mulB, CUstream stream,
                                        int NPart) {
    d_lincomb<<<g1(NPart), DROPIN_THREADS, 0, S(stream)>>>(dst, a, mulA, b, mulB, nullptr, 0.0, 0.0, 0, NPart);
    check_launch("linearCombination2Async");
}

HSB_EXPORT void linearCombination3Async(double* dst, double* a, double mulA, double* b, double mulB, double* c,
                                        double mulC, CUstream stream, int NPart) {
    d_lincomb<<<g1(NPart), DROPIN_THREADS, 0, S(stream)>>>(dst, a, mulA, b, mulB, c, mulC, 0.0, 0, NPart);
    check_launch("linearCombination3Async");
}

// ------------------------------------------------------------------ dot products (dot.cu)
__global__ void d_dotmask(double* dst, const double* ax, const double* ay, const double* az, const double* bx,
                          const double* by, const double* bz, double axm, double aym, double azm, double bxm,
                          double bym, double bzm, int n) {
    GRID_STRIDE(i, n) {
        const double a0 = axm * mu1(ax, i), a1 = aym * mu1(ay, i), a2 = azm * mu1(az, i);
        const double b0 = bxm * mu1(bx, i), b1 = bym * mu1(by, i), b2 = bzm * mu1(bz, i);
        dst[i] = a0 * b0 + a1 * b1 + a2 * b2;
    }
}

HSB_EXPORT void dotMaskAsync(double* dst, double* ax, double* ay, double* az, double* bx, double* by, double* bz,
                             double axMul, double ayMul, double azMul, double bxMul, double byMul, double bzMul,
                             CUstream stream, int Npart) {
    d_dotmask<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dst, ax, ay, az, bx, by, bz, axMul, ayMul, azMul, bxMul,
                                                           byMul, bzMul, Npart);
    check_launch("dotMaskAsync");
}

HSB_EXPORT void dotAsync(double* dst, double* ax, double* ay, double* az, double* bx, double* by, double* bz,
                         CUstream stream, int Npart) {
    d_dotmask<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dst, ax, ay, az, bx, by, bz, 1, 1, 1, 1, 1, 1, Npart);
    check_launch("dotAsync");
}

__global__ void d_dotsign(double* dst, const double* ax, const double* ay, const double* az, const double* bx,
                          const double* by, const double* bz, const double* cx, const double* cy, const double* cz,
                          int n) {
    GRID_STRIDE(i, n) {
        const double d = ax[i] * bx[i] + ay[i] * by[i] + az[i] * bz[i];
        const double s = -(bx[i] * cx[i] + by[i] * cy[i] + bz[i] * cz[i]);
        dst[i] = copysign(d, s);
    }
}

HSB_EXPORT void dotSignAsync(double* dst, double* ax, double* ay, double* az, double* bx, double* by, double* bz,
                             double* cx, double* cy, double* cz, CUstream stream, int Npart) {
    d_dotsign<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dst, ax, ay, az, bx, by, bz, cx, cy, cz, Npart);
    check_launch("dotSignAsync");
}

// ------------------------------------------------------------------ partial reductions (reduce.h)
// Each of the `blocks` blocks reduces a strided share of the N inputs into output[block];
// the caller finishes on the host (gpu/reductor.go:69-203).  Warp-shuffle trees (the
// reference's CUDPP-style volatile shared-memory tail is not used).
enum { R_SUM = 0, R_SDOT, R_MAX, R_MIN, R_MAXABS, R_MAXDIFF, R_MAXSUM, R_MAXN3, R_MAXN3D };

template <int OP>
__global__ void d_partial(const double* a, const double* b, const double* c, const double* d, const double* e,
                          const double* f, double* out, int N) {
    const bool is_sum = (OP == R_SUM || OP == R_SDOT);
    double acc = is_sum ? 0.0 : (OP == R_MIN ? INFINITY : -INFINITY);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
        double v;
        switch (OP) {
            case R_SUM: v = a[i]; break;
            case R_SDOT: v = a[i] * b[i]; break;
            case R_MAX:
            case R_MIN: v = a[i]; break;
            case R_MAXABS: v = fabs(a[i]); break;
            case R_MAXDIFF: v = fabs(a[i] - b[i]); break;
            case R_MAXSUM: v = fabs(a[i] + b[i]); break;
            case R_MAXN3: v = a[i] * a[i] + b[i] * b[i] + c[i] * c[i]; break;
            default: {
                const double x = a[i] - d[i], y = b[i] - e[i], z = c[i] - f[i];
                v = x * x + y * y + z * z;
            }
        }
        if (is_sum) acc += v;
        else if (OP == R_MIN) acc = fmin(acc, v);
        else acc = fmax(acc, v);
    }
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    acc = is_sum ? warp_sum_d(acc) : (OP == R_MIN ? warp_min_d(acc) : warp_max_d(acc));
    if (lane == 0) sh[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = sh[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); k++)
            r = is_sum ? r + sh[k] : (OP == R_MIN ? fmin(r, sh[k]) : fmax(r, sh[k]));
        // an empty block reports the neutral element of a sum, or a value that cannot win
        // the host-side max/min (the caller's maxima are of non-negative quantities)
        out[blockIdx.x] = r;
    }
}

template <int OP>
static void partial_launch(const char* who, const double* a, const double* b, const double* c, const double* d,
                           const double* e, const double* f, double* out, int blocks, int N, CUstream s) {
    if (blocks <= 0) return;
    d_partial<OP><<<blocks, DROPIN_THREADS, 0, S(s)>>>(a, b, c, d, e, f, out, N);
    check_launch(who);
}

HSB_EXPORT void partialSumAsync(double* input, double* output, int blocks, int threads, int N, CUstream s) {
    (void)threads;
    partial_launch<R_SUM>("partialSumAsync", input, 0, 0, 0, 0, 0, output, blocks, N, s);
}
HSB_EXPORT void partialSDotAsync(double* in1, double* in2, double* output, int blocks, int threads, int N, CUstream s) {
    (void)threads;
    partial_launch<R_SDOT>("partialSDotAsync", in1, in2, 0, 0, 0, 0, output, blocks, N, s);
}
HSB_EXPORT void partialMaxAsync(double* input, double* output, int blocks, int threads, int N, CUstream s) {
    (void)threads;
    partial_launch<R_MAX>("partialMaxAsync", input, 0, 0, 0, 0, 0, output, blocks, N, s);
}
HSB_EXPORT void partialMinAsync(double* input, double* output, int blocks, int threads, int N, CUstream s) {
    (void)threads;
    partial_launch<R_MIN>("partialMinAsync", input, 0, 0, 0, 0, 0, output, blocks, N, s);
}
HSB_EXPORT void partialMaxAbsAsync(double* input, double* output, int blocks, int threads, int N, CUstream s) {
    (void)threads;
    partial_launch<R_MAXABS>("partialMaxAbsAsync", input, 0, 0, 0, 0, 0, output, blocks, N, s);
}
HSB_EXPORT void partialMaxDiffAsync(double* a, double* b, double* output, int blocks, int threads, int N, CUstream s) {
    (void)threads;
    partial_launch<R_MAXDIFF>("partialMaxDiffAsync", a, b, 0, 0, 0, 0, output, blocks, N, s);
}
HSB_EXPORT void partialMaxSumAsync(double* a, double* b, double* output, int blocks, int threads, int N, CUstream s) {
    (void)threads;
    partial_launch<R_MAXSUM>("partialMaxSumAsync", a, b, 0, 0, 0, 0, output, blocks, N, s);
}
HSB_EXPORT void partialMaxNorm3SqAsync(double* x, double* y, double* z, double* output, int blocks, int threads,
                                       int N, CUstream s) {
    (void)threads;
    partial_launch<R_MAXN3>("partialMaxNorm3SqAsync", x, y, z, 0, 0, 0, output, blocks, N, s);
}
HSB_EXPORT void partialMaxNorm3SqDiffAsync(double* x1, double* y1, double* z1, double* x2, double* y2, double* z2,
                                           double* output, int blocks, int threads, int N, CUstream s) {
    (void)threads;
    partial_launch<R_MAXN3D>("partialMaxNorm3SqDiffAsync", x1, y1, z1, x2, y2, z2, output, blocks, N, s);
}

// ------------------------------------------------------------------ MFA tables
// m_e(T) and the reduced longitudinal susceptibility on T_i = Tc * i / (npts - 1), in FP64 on
// the device: m_e by the Ridders iteration of brillouinKern (brillouin.cu:88-138), chi by
// kappaKern's expression with unit masks (kappa.cu:15-61): chi = f / (1 - f) / (S/(S+1) 3 Tc),
// f = b W'(m_e b), b = S/(S+1) 3 Tc / T (multiply by Ms0^2 mu0 / (n kB), mod_kappa.go:76-89,
// for the physical value).  T = 0 gives m_e = 1, chi = 0; T >= Tc gives m_e = 0.
__global__ void d_mfa_table(double Tc, double J, int n, double* T, double* me, double* chi) {
    GRID_STRIDE(i, n) {
        const double t = (n > 1) ? Tc * (double)i / (double)(n - 1) : Tc;
        T[i] = t;
        const double preS = (J > HSB_INF_SPIN) ? 1.0 : J / (J + 1.0);
        double m = 0.0, c = 0.0;
        if (t == 0.0) {
            m = 1.0;
        } else if (t < Tc) {
            const double pre = 3.0 * preS * (Tc / t);
            const double dT = (Tc - t) / Tc;
            m = fabs(d_ridders([&](double nn) { return d_model(nn, J, pre); }, dT < 0.0004 ? -0.1 : 0.01,
                               dT < 0.0004 ? 0.5 : 1.1));
            const double b = preS * 3.0 * Tc / t;
            double f = (J > HSB_INF_SPIN) ? d_dLdx(m * b) : d_dBjdx(J, m * b);
            f = b * f;
            c = (f / (1.0 - f)) / (preS * 3.0 * Tc);
        }
        me[i] = m;
        chi[i] = c;
    }
}

// ------------------------------------------------------------------ Debye heat capacity (Cp.cu)
// Cp = n (T/Td)^3 * integral_0^{Td/T} x^4 e^x / (e^x - 1)^2 dx by the composite trapezoid
// rule on 61 intervals (the reference's INTMAXSTEPS); below T/Td = 0.01 the low-temperature
// limit n (4 pi^4 / 15) (T/Td)^3.  kB and the density multiplier are applied by the caller.
#define HSB_DEBYE_STEPS 61
__device__ __forceinline__ double d_debye_integrand(double x) {
    const double ex = exp(x);
    return (x <= HSB_ZERO) ? 0.0 : (x * x * x * x * ex) / ((ex - 1.0) * (ex - 1.0));
}

__global__ void d_cp(double* Cp, const double* T, const double* Tdm, const double* nm, double TdMul, int n) {
    GRID_STRIDE(i, n) {
        const double nn = mu1(nm, i);
        const double Td = TdMul * mu1(Tdm, i);
        const double Ti = T[i];
        if (Td == 0.0) {
            Cp[i] = 0.0;
            continue;
        }
        const double u = Td / Ti;   // upper integration limit
        const double r = Ti / Td;
        if (r < 0.01) {
            const double pi4 = M_PI * M_PI * M_PI * M_PI;
            Cp[i] = nn * (12.0 / 5.0) * (1.0 / 9.0) * pi4 * (r * r * r);
            continue;
        }
        const double h = u / (double)HSB_DEBYE_STEPS;
        double inner = 0.0, x = 0.0;
        for (int j = 1; j < HSB_DEBYE_STEPS; j++) {
            x += h;
            inner += d_debye_integrand(x);
        }
        x += h;
        const double ends = d_debye_integrand(0.0) + d_debye_integrand(x);
        const double integral = (ends + 2.0 * inner) * (0.5 * h);
        Cp[i] = nn * integral / (u * u * u);
    }
}

HSB_EXPORT void cpAsync(double* Cp, double* T, double* Td, double* n, const double TdMul, const int Npart,
                        CUstream stream) {
    d_cp<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(Cp, T, Td, n, TdMul, Npart);
    check_launch("cpAsync");
}

// ------------------------------------------------------------------ spin temperature (Ts.cu)
// The temperature at which the mean-field equilibrium magnetization equals msat / Msat0T0:
// solve B_S(S^2 J0 m / T) = m for T in [0, Tc] (J0 = 3 Tc / (S (S + 1))) with the same
// Ridders iteration as brillouinAsync.  Msat0T0 = 0 -> 0, msat = Msat0T0 -> 0, msat = 0 -> Tc.
__device__ double d_ts_model(double T, double S_, double pre, double m) {
    const double x = (T == 0.0) ? 1.0e38 : pre / T;
    return d_Bj(S_, x) - m;
}

__global__ void d_ts(double* Ts, const double* msm, const double* ms0T0m, const double* Tcm, const double* Sm,
                     double msMul, double ms0T0Mul, double TcMul, double SMul, int n) {
    GRID_STRIDE(i, n) {
        const double ms0T0 = ms0T0Mul * mu1(ms0T0m, i);
        if (ms0T0 == 0.0) {
            Ts[i] = 0.0;
            continue;
        }
        const double ms = msMul * mu1(msm, i);
        if (ms == ms0T0) {
            Ts[i] = 0.0;
            continue;
        }
        const double Tc = TcMul * mu1(Tcm, i);
        if (ms == 0.0) {
            Ts[i] = Tc;
            continue;
        }
        const double Sp = SMul * mu1(Sm, i);
        const double J0 = 3.0 * Tc / (Sp * (Sp + 1.0));
        const double m = ms / ms0T0;
        const double pre = Sp * Sp * J0 * m;
        Ts[i] = d_ridders([&](double T) { return d_ts_model(T, Sp, pre, m); }, 0.0, Tc);
    }
}

HSB_EXPORT void tsAsync(double* Ts, double* msat, double* msat0T0, double* Tc, double* S_, const double msatMul,
                        const double msat0T0Mul, const double TcMul, const double SMul, int Npart, CUstream stream) {
    d_ts<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(Ts, msat, msat0T0, Tc, S_, msatMul, msat0T0Mul, TcMul, SMul,
                                                      Npart);
    check_launch("tsAsync");
}

// ------------------------------------------------------------------ weighted average (wavg.cu)
// dst = (w0 a + w1 b + 2 R sqrt(w0 a w1 b)) / (w0 + w1 + 2 R sqrt(w0 w1)), 0 where the
// denominator vanishes.
__global__ void d_wavg(double* dst, const double* a, const double* b, const double* w0m, const double* w1m,
                       const double* Rm, double w0Mul, double w1Mul, double RMul, int n) {
    GRID_STRIDE(i, n) {
        const double w0 = w0Mul * mu1(w0m, i), w1 = w1Mul * mu1(w1m, i), R = RMul * mu1(Rm, i);
        const double x0 = a[i], x1 = b[i];
        const double den = w0 + w1 + 2.0 * R * sqrt(w0 * w1);
        dst[i] = (den == 0.0) ? 0.0 : (w0 * x0 + w1 * x1 + 2.0 * R * sqrt(w0 * x0 * w1 * x1)) / den;
    }
}

HSB_EXPORT void wavgAsync(double* dst, double* a, double* b, double* w0, double* w1, double* R, double w0Mul,
                          double w1Mul, double RMul, CUstream stream, int Npart) {
    d_wavg<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(dst, a, b, w0, w1, R, w0Mul, w1Mul, RMul, Npart);
    check_launch("wavgAsync");
}

// ------------------------------------------------------------------ energy flow (energy_flow.cu)
// w = Tc S^2 n / (S (S + 1)) (m . R), with Tc and n taken from their masks alone (the
// reference applies no multiplier to them) and 0 where n, S or Tc vanishes.
__global__ void d_energy_flow(double* w, const double* mx, const double* my, const double* mz, const double* Rx,
                              const double* Ry, const double* Rz, const double* Tcm, const double* Sm,
                              const double* nm, double SMul, int n) {
    GRID_STRIDE(i, n) {
        const double Sp = SMul * mu1(Sm, i), Tc = mu1(Tcm, i), nn = mu1(nm, i);
        if (nn == 0.0 || Sp == 0.0 || Tc == 0.0) {
            w[i] = 0.0;
            continue;
        }
        const double mR = mx[i] * Rx[i] + my[i] * Ry[i] + mz[i] * Rz[i];
        w[i] = (Tc * Sp * Sp * nn / (Sp * (Sp + 1.0))) * mR;
    }
}

HSB_EXPORT void energyFlowAsync(double* w, double* mx, double* my, double* mz, double* Rx, double* Ry, double* Rz,
                                double* Tc, double* S_, double* n, double SMul, int Npart, CUstream stream) {
    d_energy_flow<<<g1(Npart), DROPIN_THREADS, 0, S(stream)>>>(w, mx, my, mz, Rx, Ry, Rz, Tc, S_, n, SMul, Npart);
    check_launch("energyFlowAsync");
}

// ------------------------------------------------------------------ nonlocal damping (llbar-nonlocal00nc.cu)
// t_c = -sum over the 6 neighbours of lambda_c / cs_d^2 ((l1 H1 + l2 H2) - H0 (l1 + l2)),
// l1, l2 = harmonic means of the cell's and the neighbour's lambda_e mask (per component),
// clamp / wrap boundaries; 0 where Msat0T0 = 0.  Neighbour indices are the grid's own in every
// direction (the reference's a1 + 1 neighbour is computed with N1 in place of N2, which
// differs from this only when N1 != N2).
__global__ void d_nonlocal00nc(double* tx, double* ty, double* tz, const double* hx, const double* hy,
                               const double* hz, const double* ms0T0m, const double* lxx, const double* lyy,
                               const double* lzz, double Lx, double Ly, double Lz, int s0, int s1, int s2,
                               double c0, double c1, double c2, int p0, int p1, int p2) {
    const long n = (long)s0 * s1 * s2;
    GRID_STRIDE(I, n) {
        if (mu1(ms0T0m, I) == 0.0) {
            tx[I] = ty[I] = tz[I] = 0.0;
            continue;
        }
        const int k = (int)(I % s2);
        const int j = (int)((I / s2) % s1);
        const int i = (int)(I / ((long)s1 * s2));
        const double* L[3] = {lxx, lyy, lzz};
        const double* H[3] = {hx, hy, hz};
        const double mul[3] = {Lx, Ly, Lz};
        const long nb[3][2] = {
            {((long)nb_lo(i, s0, p0) * s1 + j) * s2 + k, ((long)nb_hi(i, s0, p0) * s1 + j) * s2 + k},
            {((long)i * s1 + nb_lo(j, s1, p1)) * s2 + k, ((long)i * s1 + nb_hi(j, s1, p1)) * s2 + k},
            {((long)i * s1 + j) * s2 + nb_lo(k, s2, p2), ((long)i * s1 + j) * s2 + nb_hi(k, s2, p2)}};
        const double inv_cs2[3] = {c0, c1, c2};
        double out[3];
        for (int c = 0; c < 3; c++) {
            const double l0 = mu1(L[c], I), H0 = H[c][I];
            double R = 0.0;
            for (int d = 0; d < 3; d++) {
                const double la = harm0(l0, mu1(L[c], nb[d][0])), lb = harm0(l0, mu1(L[c], nb[d][1]));
                R += mul[c] * inv_cs2[d] * ((la * H[c][nb[d][0]] + lb * H[c][nb[d][1]]) - H0 * (la + lb));
            }
            out[c] = -R;
        }
        tx[I] = out[0];
        ty[I] = out[1];
        tz[I] = out[2];
    }
}

HSB_EXPORT void llbar_nonlocal00nc_async(double* tx, double* ty, double* tz, double* hx, double* hy, double* hz,
                                         double* msat0T0, double* lambda_e_xx, double* lambda_e_yy,
                                         double* lambda_e_zz, const double lambda_eMul_xx,
                                         const double lambda_eMul_yy, const double lambda_eMul_zz, const int sx,
                                         const int sy, const int sz, const double csx, const double csy,
                                         const double csz, const int pbc_x, const int pbc_y, const int pbc_z,
                                         CUstream stream) {
    const long n = (long)sx * sy * sz;
    d_nonlocal00nc<<<g1(n), DROPIN_THREADS, 0, S(stream)>>>(
        tx, ty, tz, hx, hy, hz, msat0T0, lambda_e_xx, lambda_e_yy, lambda_e_zz, lambda_eMul_xx, lambda_eMul_yy,
        lambda_eMul_zz, sx, sy, sz, 1.0 / (csx * csx), 1.0 / (csy * csy), 1.0 / (csz * csz), pbc_x, pbc_y, pbc_z);
    check_launch("llbar_nonlocal00nc_async");
}


HSB_EXPORT int hsb_mfa_table(double Tc, double J, int npts, double* T_host, double* me_host, double* chi_host) {
    if (!(Tc > 0) || !(J > 0) || npts < 1 || !T_host || !me_host || !chi_host) {
        hsb_set_error("hsb_mfa_table: bad argument");
        return HSB_ERR_INVALID;
    }
    double* d = nullptr;
    HSB_CUDA_TRY(cudaMalloc(&d, sizeof(double) * 3 * npts));
    d_mfa_table<<<g1(npts), DROPIN_THREADS>>>(Tc, J, npts, d, d + npts, d + 2 * npts);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(T_host, d, sizeof(double) * npts, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(me_host, d + npts, sizeof(double) * npts, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(chi_host, d + 2 * npts, sizeof(double) * npts, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        hsb_set_error("hsb_mfa_table: %s", cudaGetErrorString(e));
        return HSB_ERR_CUDA;
    }
    return HSB_OK;
}

// m_e at one temperature: linear interpolation in a 1024-point FP64 table (cached per
// (Tc, J) in the caller's memory is not needed: the table costs one small kernel).
HSB_EXPORT int hsb_mfa_equilibrium(double T, double Tc, double J, double* me) {
    if (!me || !(T >= 0)) {
        hsb_set_error("hsb_mfa_equilibrium: bad argument");
        return HSB_ERR_INVALID;
    }
    if (T >= Tc) {
        *me = 0.0;
        return HSB_OK;
    }
    const int n = 1024;
    static double Tt[1024], mt[1024], ct[1024];
    int rc = hsb_mfa_table(Tc, J, n, Tt, mt, ct);
    if (rc != HSB_OK) return rc;
    const double x = T / Tc * (n - 1);
    int i = (int)x;
    if (i >= n - 1) i = n - 2;
    const double f = x - i;
    *me = mt[i] + f * (mt[i + 1] - mt[i]);
    return HSB_OK;
}
