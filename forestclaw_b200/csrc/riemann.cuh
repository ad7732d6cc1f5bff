// riemann.cuh -- __device__ Riemann solvers of the B200 package.
//
// Each solver is a struct with compile-time sizes and two device functions that
// act on ONE interface (the per-interface body of the reference's loop over
// i = 2-mbc..mx+mbc), so the fused update kernel can give every interface its
// own thread.  Arithmetic follows the cited Fortran line by line, in the same
// evaluation order, so that with FMA contraction disabled the FP64 instantiation
// reproduces the FP64 CPU path bit for bit.
//
//   rpn2(ixy, qL, qR, auxL, auxR) -> wave[mw][m], s[mw], amdq[m], apdq[m], extra
//       qL = state of cell i-1 (qr(i-1,:)), qR = state of cell i (ql(i,:)),
//       auxL/auxR = aux of cells i-1 / i on the sweep line (the reference passes aux2 for both).
//   rpt2(ixy, imp, qL, qR, aux1, aux2, aux3, extra, asdq) -> bmasdq[m], bpasdq[m]
//       aux1/2/3 = aux of cell i1 = i-2+imp on the lines below / on / above the sweep line.
#pragma once
#include <cuda_runtime.h>

namespace fcb {

template <typename T> __device__ __forceinline__ T dmin1(T a, T b) { return a < b ? a : b; }
template <typename T> __device__ __forceinline__ T dmax1(T a, T b) { return a > b ? a : b; }
template <typename T> __device__ __forceinline__ T sgn1(T x) { return copysign(T(1), x); }

// ---------------------------------------------------------------------------
// Scalar advection with edge velocities in aux(:,:,1:2).
// applications/clawpack/advection/2d/all/clawpack46_rpn2adv.f, clawpack46_rpt2adv.f
// ---------------------------------------------------------------------------
struct RPAdvection {
    static constexpr int MEQN = 1, MWAVES = 1, MAUX = 2, NEXTRA = 1;
    static constexpr bool CONS_FLUX = false;
    __device__ static void flux64(int ixy, const double* q, double grav, double* f) { (void)ixy; (void)grav; f[0] = q[0]; }
    // FP64 Godunov split for the FP32-wave path
    __device__ static void godunov64(int ixy, const double* qL, const double* qR, const double* aL, const double* aR,
                                     const double* fL, const double* fR, const float* ap32, double* am, double* ap,
                                     double grav)
    {
        (void)aL; (void)fL; (void)fR; (void)ap32; (void)grav;
        const double s = aR[ixy - 1], d = qR[0] - qL[0];
        am[0] = 0.0 + dmin1(s, 0.0) * d;
        ap[0] = 0.0 + dmax1(s, 0.0) * d;
    }
    template <typename T>
    __device__ static void rpn2(int ixy, const T* qL, const T* qR, const T* auxL, const T* auxR,
                                T wave[MWAVES][MEQN], T s[MWAVES], T amdq[MEQN], T apdq[MEQN],
                                T extra[NEXTRA], T grav)
    {
        (void)auxL; (void)grav; (void)extra;
        T delta = qR[0] - qL[0];
        wave[0][0] = delta;
        s[0] = auxR[ixy - 1];                       // s(i,mw) = auxl(i,iface)
        amdq[0] = T(0) + dmin1(s[0], T(0)) * wave[0][0];
        apdq[0] = T(0) + dmax1(s[0], T(0)) * wave[0][0];
    }
    template <typename T>
    __device__ static void rpt2(int ixy, int imp, const T* qL, const T* qR, const T* aux1, const T* aux2,
                                const T* aux3, const T extra[NEXTRA], const T* asdq, T* bm, T* bp, T grav, T drytol)
    {
        (void)imp; (void)qL; (void)qR; (void)aux1; (void)extra; (void)grav; (void)drytol;
        const int kv = 3 - ixy;
        bm[0] = dmin1(aux2[kv - 1], T(0)) * asdq[0];
        bp[0] = dmax1(aux3[kv - 1], T(0)) * asdq[0];
    }
};

// ---------------------------------------------------------------------------
// Shallow water, Roe solver with Harten-Hyman entropy fix.
// applications/clawpack/shallow/2d/rp/clawpack46_rpn2.f:1-247, clawpack46_rpt2.f:248-321
// extra = Roe averages (u, v, a) of the interface (the common block /comroe/).
// ---------------------------------------------------------------------------
struct RPShallowRoe {
    static constexpr int MEQN = 3, MWAVES = 3, MAUX = 0, NEXTRA = 3;
    static constexpr bool CONS_FLUX = true;
    // normal flux in direction ixy, FP64 (one division per cell)
    __device__ static void flux64(int ixy, const double* q, double grav, double* f)
    {
        const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
        const double h = q[0], inv = 1.0 / h;
        f[0] = q[mu];
        f[mu] = q[mu] * q[mu] * inv + 0.5 * grav * h * h;
        f[mv] = q[mu] * q[mv] * inv;
    }
    // amdq as the FP64 remainder of the flux difference: amdq + apdq = f(qR) - f(qL)
    __device__ static void godunov64(int ixy, const double* qL, const double* qR, const double* aL, const double* aR,
                                     const double* fL, const double* fR, const float* ap32, double* am, double* ap,
                                     double grav)
    {
        (void)ixy; (void)qL; (void)qR; (void)aL; (void)aR; (void)grav;
        for (int m = 0; m < 3; m++) { ap[m] = (double)ap32[m]; am[m] = (fR[m] - fL[m]) - ap[m]; }
    }
    template <typename T>
    __device__ static void rpn2(int ixy, const T* qL, const T* qR, const T* auxL, const T* auxR,
                                T wave[MWAVES][MEQN], T s[MWAVES], T amdq[MEQN], T apdq[MEQN],
                                T extra[NEXTRA], T grav)
    {
        (void)auxL; (void)auxR;
        const int mu = (ixy == 1) ? 1 : 2;   // 0-based component of the normal momentum
        const int mv = (ixy == 1) ? 2 : 1;
        // :91-99
        T h = (qL[0] + qR[0]) / T(2);
        T hsqrtl = sqrt(qL[0]);
        T hsqrtr = sqrt(qR[0]);
        T hsq2 = hsqrtl + hsqrtr;
        T u = (qL[mu] / hsqrtl + qR[mu] / hsqrtr) / hsq2;
        T v = (qL[mv] / hsqrtl + qR[mv] / hsqrtr) / hsq2;
        T a = sqrt(grav * h);
        extra[0] = u; extra[1] = v; extra[2] = a;
        // :105-129
        T d1 = qR[0] - qL[0];
        T d2 = qR[mu] - qL[mu];
        T d3 = qR[mv] - qL[mv];
        T a1 = ((u + a) * d1 - d2) / (T(2) * a);
        T a2 = -(v * d1) + d3;
        T a3 = (-((u - a) * d1) + d2) / (T(2) * a);
        wave[0][0] = a1; wave[0][mu] = a1 * (u - a); wave[0][mv] = a1 * v; s[0] = u - a;
        wave[1][0] = T(0); wave[1][mu] = T(0); wave[1][mv] = a2; s[1] = u;
        wave[2][0] = a3; wave[2][mu] = a3 * (u + a); wave[2][mv] = a3 * v; s[2] = u + a;
        // entropy fix :170-229
        do {
            T him1 = qL[0];
            T s0 = qL[mu] / him1 - sqrt(grav * him1);
            if (s0 > T(0) && s[0] > T(0)) {
                amdq[0] = T(0); amdq[1] = T(0); amdq[2] = T(0);
                break;
            }
            T h1 = qL[0] + wave[0][0];
            T hu1 = qL[mu] + wave[0][mu];
            T s1 = hu1 / h1 - sqrt(grav * h1);
            T sfract;
            if (s0 < T(0) && s1 > T(0)) sfract = s0 * ((s1 - s[0]) / (s1 - s0));
            else if (s[0] < T(0)) sfract = s[0];
            else sfract = T(0);
            for (int m = 0; m < 3; m++) amdq[m] = sfract * wave[0][m];
            if (s[1] > T(0)) break;
            for (int m = 0; m < 3; m++) amdq[m] = amdq[m] + s[1] * wave[1][m];
            T hi = qR[0];
            T s03 = qR[mu] / hi + sqrt(grav * hi);
            T h3 = qR[0] - wave[2][0];
            T hu3 = qR[mu] - wave[2][mu];
            T s3 = hu3 / h3 + sqrt(grav * h3);
            if (s3 < T(0) && s03 > T(0)) sfract = s3 * ((s03 - s[2]) / (s03 - s3));
            else if (s[2] < T(0)) sfract = s[2];
            else break;
            for (int m = 0; m < 3; m++) amdq[m] = amdq[m] + sfract * wave[2][m];
        } while (0);
        // :234-242
        for (int m = 0; m < 3; m++) {
            T df = T(0);
            for (int mw = 0; mw < 3; mw++) df = df + s[mw] * wave[mw][m];
            apdq[m] = df - amdq[m];
        }
    }
    template <typename T>
    __device__ static void rpt2(int ixy, int imp, const T* qL, const T* qR, const T* aux1, const T* aux2,
                                const T* aux3, const T extra[NEXTRA], const T* asdq, T* bm, T* bp, T grav, T drytol)
    {
        (void)imp; (void)qL; (void)qR; (void)aux1; (void)aux2; (void)aux3; (void)grav; (void)drytol;
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        T u = extra[0], v = extra[1], a = extra[2];
        T a1 = ((v + a) * asdq[0] - asdq[mv]) / (T(2) * a);
        T a2 = asdq[mu] - u * asdq[0];
        T a3 = (-((v - a) * asdq[0]) + asdq[mv]) / (T(2) * a);
        T wb[3][3];   // wb[mw][m]
        T sb[3];
        wb[0][0] = a1; wb[0][mu] = a1 * u; wb[0][mv] = a1 * (v - a); sb[0] = v - a;
        wb[1][0] = T(0); wb[1][mu] = a2; wb[1][mv] = T(0); sb[1] = v;
        wb[2][0] = a3; wb[2][mu] = a3 * u; wb[2][mv] = a3 * (v + a); sb[2] = v + a;
        for (int m = 0; m < 3; m++) {
            T b1 = T(0), b2 = T(0);
            for (int mw = 0; mw < 3; mw++) {
                b1 = b1 + dmin1(sb[mw], T(0)) * wb[mw][m];
                b2 = b2 + dmax1(sb[mw], T(0)) * wb[mw][m];
            }
            bm[m] = b1; bp[m] = b2;
        }
    }
};

// ---------------------------------------------------------------------------
// Shallow water f-waves with bathymetry b = aux(:,:,1).
// applications/clawpack/shallow/2d/rp/rpn2_tsunami.f90:3-222, rpt2_tsunami.f90:3-170
// ---------------------------------------------------------------------------
struct RPShallowFWave {
    static constexpr int MEQN = 3, MWAVES = 3, MAUX = 1, NEXTRA = 1;
    static constexpr bool CONS_FLUX = true;
    // normal flux in direction ixy, FP64 (one division per cell)
    __device__ static void flux64(int ixy, const double* q, double grav, double* f)
    {
        const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
        const double h = q[0], inv = 1.0 / h;
        f[0] = q[mu];
        f[mu] = q[mu] * q[mu] * inv + 0.5 * grav * h * h;
        f[mv] = q[mu] * q[mv] * inv;
    }
    // f-waves sum to the flux difference plus the bathymetry source g*hbar*(bR-bL)
    __device__ static void godunov64(int ixy, const double* qL, const double* qR, const double* aL, const double* aR,
                                     const double* fL, const double* fR, const float* ap32, double* am, double* ap,
                                     double grav)
    {
        const int mu = (ixy == 1) ? 1 : 2;
        for (int m = 0; m < 3; m++) {
            double fd = fR[m] - fL[m];
            if (m == mu) fd = fd + grav * (0.5 * (qR[0] + qL[0])) * (aR[0] - aL[0]);
            ap[m] = (double)ap32[m];
            am[m] = fd - ap[m];
        }
    }
    template <typename T>
    __device__ static void rpn2(int ixy, const T* qL, const T* qR, const T* auxL, const T* auxR,
                                T fwave[MWAVES][MEQN], T s[MWAVES], T amdq[MEQN], T apdq[MEQN],
                                T extra[NEXTRA], T grav)
    {
        (void)extra;
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        T hL = qL[0], hR = qR[0];
        T huL = qL[mu], huR = qR[mu];
        T bL = auxL[0], bR = auxR[0];
        T hvL = qL[mv], hvR = qR[mv];
        T uR = huR / hR, vR = hvR / hR;
        T phiR = T(0.5) * grav * (hR * hR) + (huR * huR) / hR;
        T uL = huL / hL, vL = hvL / hL;
        T phiL = T(0.5) * grav * (hL * hL) + (huL * huL) / hL;
        T uhat = (sqrt(grav * hL) * uL + sqrt(grav * hR) * uR) / (sqrt(grav * hR) + sqrt(grav * hL));
        T chat = sqrt(grav * T(0.5) * (hR + hL));
        T hbar = T(0.5) * (hR + hL);
        T fd1 = (hR * uR) - (hL * uL);
        T fd2 = phiR - phiL + grav * hbar * (bR - bL);
        T fd3 = hR * uR * vR - hL * uL * vL;
        T s1 = fmin(uL - sqrt(grav * hL), uhat - chat);
        T s3 = fmax(uR + sqrt(grav * hR), uhat + chat);
        T s2 = T(0.5) * (s1 + s3);
        T b1 = -(fd2 - s3 * fd1) / (s3 - s1);
        T b3 = (fd2 - s1 * fd1) / (s3 - s1);
        T b2 = fd3 - b1 * vL - b3 * vR;
        T fw[3][3];   // fw[row][wave], rows (h, normal, transverse)
        fw[0][0] = b1; fw[1][0] = b1 * s1; fw[2][0] = b1 * vL;
        fw[0][1] = T(0); fw[1][1] = T(0); fw[2][1] = b2;
        fw[0][2] = b3; fw[1][2] = b3 * s3; fw[2][2] = b3 * vR;
        s[0] = s1; s[1] = s2; s[2] = s3;
        for (int mw = 0; mw < 3; mw++) {
            fwave[mw][0] = fw[0][mw];
            fwave[mw][mu] = fw[1][mw];
            fwave[mw][mv] = fw[2][mw];
        }
        T szm[3], szp[3];
        for (int mw = 0; mw < 3; mw++) {
            T z = sgn1(s[mw]);
            szm[mw] = (T(1) - z) / T(2);
            szp[mw] = (T(1) + z) / T(2);
        }
        for (int m = 0; m < 3; m++) {
            T am = szm[0] * fwave[0][m];
            am = am + szm[1] * fwave[1][m];
            am = am + szm[2] * fwave[2][m];
            T ap = szp[0] * fwave[0][m];
            ap = ap + szp[1] * fwave[1][m];
            ap = ap + szp[2] * fwave[2][m];
            amdq[m] = am; apdq[m] = ap;
        }
    }
    template <typename T>
    __device__ static void rpt2(int ixy, int imp, const T* qL, const T* qR, const T* aux1, const T* aux2,
                                const T* aux3, const T extra[NEXTRA], const T* asdq, T* bm, T* bp, T g, T tol)
    {
        (void)extra;
        const int mu = (ixy == 1) ? 1 : 2;
        const int mv = (ixy == 1) ? 2 : 1;
        T hl = qL[0], hr = qR[0];
        T hul = qL[mu], hur = qR[mu];
        T hvl = qL[mv], hvr = qR[mv];
        T ul, vl, ur, vr;
        if (hl < tol) { hl = T(0); ul = T(0); vl = T(0); } else { ul = hul / hl; vl = hvl / hl; }
        if (hr < tol) { hr = T(0); ur = T(0); vr = T(0); } else { ur = hur / hr; vr = hvr / hr; }
        T sv[3] = {T(0), T(0), T(0)}, beta[3] = {T(0), T(0), T(0)};
        T r[3][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}, {T(0), T(0), T(0)}};   // r[m][mw]
        bool skip = (hl <= tol && hr <= tol);
        if (!skip) {
            T eta = (imp == 1) ? qL[0] + aux2[0] : qR[0] + aux2[0];
            if (eta < fmax(aux1[0], aux3[0])) skip = true;
        }
        if (!skip) {
            T vhat = (vr * sqrt(hr)) / (sqrt(hr) + sqrt(hl)) + (vl * sqrt(hl)) / (sqrt(hr) + sqrt(hl));
            T uhat = (ur * sqrt(hr)) / (sqrt(hr) + sqrt(hl)) + (ul * sqrt(hl)) / (sqrt(hr) + sqrt(hl));
            T hhat = (hr + hl) / T(2);
            T roe1 = vhat - sqrt(g * hhat);
            T roe3 = vhat + sqrt(g * hhat);
            T s1l = vl - sqrt(g * hl);
            T s3r = vr + sqrt(g * hr);
            T s1 = fmin(roe1, s1l);
            T s3 = fmax(roe3, s3r);
            T s2 = uhat;
            sv[0] = s1; sv[1] = s2; sv[2] = s3;
            T delf1 = asdq[0], delf2 = asdq[mu], delf3 = asdq[mv];
            beta[0] = (s3 * delf1 / (s3 - s1)) - (delf3 / (s3 - s1));
            beta[1] = -(s2 * delf1) + delf2;
            beta[2] = (delf3 / (s3 - s1)) - (s1 * delf1 / (s3 - s1));
            r[0][0] = T(1); r[mu][0] = s2; r[mv][0] = s1;
            r[0][1] = T(0); r[mu][1] = T(1); r[mv][1] = T(0);
            r[0][2] = T(1); r[mu][2] = s2; r[mv][2] = s3;
        }
        T szm[3], szp[3];
        for (int mw = 0; mw < 3; mw++) {
            T z = sgn1(sv[mw]);
            szm[mw] = (T(1) - z) / T(2) * sv[mw] * beta[mw];
            szp[mw] = (T(1) + z) / T(2) * sv[mw] * beta[mw];
        }
        for (int m = 0; m < 3; m++) {
            T b1 = szm[0] * r[m][0];
            b1 = b1 + szm[1] * r[m][1];
            b1 = b1 + szm[2] * r[m][2];
            T b2 = szp[0] * r[m][0];
            b2 = b2 + szp[1] * r[m][1];
            b2 = b2 + szp[2] * r[m][2];
            bm[m] = b1; bp[m] = b2;
        }
    }
};

// clawpack46_inlinelimiter.f:59-104
template <typename T>
__device__ __forceinline__ T limiter_phi(int mthlim, T r)
{
    switch (mthlim) {
    case 1: return dmax1(T(0), dmin1(T(1), r));
    case 2: return dmax1(dmax1(T(0), dmin1(T(1), T(2) * r)), dmin1(T(2), r));
    case 3: return (r + fabs(r)) / (T(1) + fabs(r));
    case 4: { T c = (T(1) + r) / T(2); return dmax1(T(0), dmin1(dmin1(c, T(2)), T(2) * r)); }
    case 5: return r;
    case 6: { T th = T((double)1.3f); return dmax1(T(0), dmin1(dmin1(th * r, (T(1) + r) / T(2)), th)); }
    default: return T(1);
    }
}

}  // namespace fcb
