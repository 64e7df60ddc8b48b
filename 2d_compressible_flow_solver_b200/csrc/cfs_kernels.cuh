// Stage, immersed-boundary, reduction and layout kernels, templated over an
// arithmetic policy.  Included by kernels_exact.cu (built with -fmad=false, so
// PolExact keeps the reference's rounding sequence) and kernels_fast.cu (FMA
// contraction on: PolF64, PolF32).
#pragma once
#include <cuda_runtime.h>
#include <cfloat>
#include <cstdint>

#include "cfs_layout.h"

namespace cfs {

// ---------------------------------------------------------------- policies
// T = storage type of the state, C = type of the WENO/HLL arithmetic.
struct PolExact { using T = double; using C = double; static constexpr bool kExact = true;  static constexpr bool kMixed = false; };
struct PolF64   { using T = double; using C = double; static constexpr bool kExact = false; static constexpr bool kMixed = false; };
struct PolF32   { using T = float;  using C = float;  static constexpr bool kExact = false; static constexpr bool kMixed = true;  };

enum { kRkTvd2 = 0, kRkTvd3Ref = 1, kRkSsp3 = 2 };
enum { kHllReference = 0, kHllDavis = 1 };

// Reconstructed face state: conserved variables, pressure, sound speed and
// (throughput forms) 1/rho.
template <class C> struct Face5 { C r, mx, my, E, p, a, ri; };

// FP32 reciprocal and reciprocal square root of the throughput forms: the
// PTX approximations themselves (one MUFU instruction each, maximum error
// 1 ulp for rcp.approx and 2 ulp for rsqrt.approx per the PTX ISA), with
// subnormal inputs and results flushed to zero.  The state's magnitudes are
// far from the subnormal range, and the row march is bound by instruction
// issue, so no range handling is wrapped around them.
__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt_fast(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ double rcp_fast(double x) { return 1.0 / x; }

// FP64 reciprocal and square root of the FP64 throughput form, from the
// hardware approximations (relative error about 2^-20 on B200, measured over
// 2^30 random arguments in [2^-40, 2^40]) refined by ONE cubically
// convergent step each, from the series of (1 - e)^-1 and (1 - e)^-1/2 in the
// approximation's residual e (an initial relative error e becomes about e^3,
// far below FP64 rounding), as fused multiply-adds.  Measured against the
// IEEE operations over the same 2^30 arguments: the reciprocal within 1 ulp,
// the square root equal in every case (two quadratic Newton-Raphson steps
// instead cost one more dependent multiply-add for the reciprocal and three
// more operations for the square root).  Inputs are finite, nonzero and normal
// where these are used (WENO weight sums >= eps^2, densities and pressures of
// physical states); a zero or negative argument yields NaN where the IEEE
// operation would give an infinity or NaN, which the callers treat alike
// (non-admissible state, a blow-up the CFL reduction reports).
//   reciprocal: e = 1 - x r, r <- r (1 + e + e^2);
//   square root: e = 1 - x y^2 for the reciprocal square root y,
//     y <- y (1 + e/2 + 3 e^2/8), then s = x y corrected once by
//     s <- s + (y/2)(x - s^2).
__device__ __forceinline__ double rcp_pos(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double e = fma(-x, r, 1.0);
    return fma(r, fma(e, e, e), r);
}
__device__ __forceinline__ double sqrt_pos(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x * y, y, 1.0);
    y = fma(y, e * fma(e, 0.375, 0.5), y);
    const double sq = x * y;
    return fma(0.5 * y, fma(-sq, sq, x), sq);
}
__device__ __forceinline__ float rcp_pos(float x) { return rcp_fast(x); }
__device__ __forceinline__ float sqrt_fast(float x) { return x * rsqrt_fast(x); }
__device__ __forceinline__ double sqrt_fast(double x) { return sqrt(x); }

// One cell's four stored variables in vector accesses (one 16-byte access in
// FP32, two in FP64; cells are 16- / 32-byte aligned in the interleaved layout).
template <class T>
__device__ __forceinline__ void ld_cell(const T* U, long long cell, T v[kVars]) {
    if constexpr (sizeof(T) == 4) {
        const float4 t = *reinterpret_cast<const float4*>(U + Layout::at(cell, 0));
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    } else {
        const double2* q = reinterpret_cast<const double2*>(U + Layout::at(cell, 0));
        const double2 a = q[0], b = q[1];
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
}
template <class T>
__device__ __forceinline__ void st_cell(T* U, long long cell, const T v[kVars]) {
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(U + Layout::at(cell, 0)) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        double2* q = reinterpret_cast<double2*>(U + Layout::at(cell, 0));
        q[0] = make_double2(v[0], v[1]);
        q[1] = make_double2(v[2], v[3]);
    }
}

// State storage: FP64 holds the value; FP32 holds value - L.off[v].
template <class T>
__device__ __forceinline__ double dec(T stored, const Layout& L, int v) {
    if constexpr (sizeof(T) == 4) return double(stored) + double(L.off[v]);
    else return double(stored);
}
template <class T, class C>
__device__ __forceinline__ C decc(T stored, const Layout& L, int v) {
    if constexpr (sizeof(T) == 4) return C(stored) + C(L.off[v]);
    else return C(stored);
}
template <class T>
__device__ __forceinline__ T enc(double value, const Layout& L, int v) {
    if constexpr (sizeof(T) == 4) return T(value - double(L.off[v]));
    else return T(value);
}

// std::min / std::max as the reference uses them (RiemmanSolverHLL.cpp:41-42):
// the first argument is returned unless the second compares smaller (larger),
// so a NaN second argument is dropped.
// Packed FP32 (sm_100 FFMA2 / FADD2 / FMUL2: two independent FP32 operations
// per instruction, each rounded as its scalar form).
__device__ __forceinline__ float2 p2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, p2(-1.0f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <class C> __device__ __forceinline__ C min_ref(C a, C b) { return (b < a) ? b : a; }
template <class C> __device__ __forceinline__ C max_ref(C a, C b) { return (a < b) ? b : a; }

// ------------------------------------------------------------------- WENO5
// Weno5th::weno5Interpolation (Weno5th.cpp:4-28) in its own operation order.
__device__ __forceinline__ double weno5_ref(double v0, double v1, double v2, double v3, double v4, double eps) {
    double beta0 = (13.0 / 12.0) * ((v0 - 2 * v1 + v2) * (v0 - 2 * v1 + v2))
                 + 0.25 * ((v0 - 4 * v1 + 3 * v2) * (v0 - 4 * v1 + 3 * v2));
    double beta1 = (13.0 / 12.0) * ((v1 - 2 * v2 + v3) * (v1 - 2 * v2 + v3))
                 + 0.25 * ((v1 - v3) * (v1 - v3));
    double beta2 = (13.0 / 12.0) * ((v2 - 2 * v3 + v4) * (v2 - 2 * v3 + v4))
                 + 0.25 * ((3 * v2 - 4 * v3 + v4) * (3 * v2 - 4 * v3 + v4));
    double alpha0 = 0.1 / ((eps + beta0) * (eps + beta0));
    double alpha1 = 0.6 / ((eps + beta1) * (eps + beta1));
    double alpha2 = 0.3 / ((eps + beta2) * (eps + beta2));
    double sum_alpha = alpha0 + alpha1 + alpha2;
    double omega0 = alpha0 / sum_alpha;
    double omega1 = alpha1 / sum_alpha;
    double omega2 = alpha2 / sum_alpha;
    return omega0 * (v0 / 3.0 - 7.0 * v1 / 6.0 + 11.0 * v2 / 6.0)
         + omega1 * (-v1 / 6.0 + 5.0 * v2 / 6.0 + v3 / 3.0)
         + omega2 * (v2 / 3.0 + 5.0 * v3 / 6.0 - v4 / 6.0);
}

// The same reconstruction with one division: alpha_k = d_k / q_k with
// q_k = (eps + beta_k)^2 is scaled by q0 q1 q2, so
// result = (sum d_k q_l q_m P_k) / (6 sum d_k q_l q_m), P_k = 6 x candidate k.
// In FP32 beta is capped at 1e9 so that the q products stay finite.
template <class C>
__device__ __forceinline__ C weno5_fast(C v0, C v1, C v2, C v3, C v4, C eps) {
    const C k13 = C(13.0 / 12.0), k14 = C(0.25);
    const C d0 = v0 - C(2) * v1 + v2, e0 = v0 - C(4) * v1 + C(3) * v2;
    const C d1 = v1 - C(2) * v2 + v3, e1 = v1 - v3;
    const C d2 = v2 - C(2) * v3 + v4, e2 = C(3) * v2 - C(4) * v3 + v4;
    C b0 = k13 * d0 * d0 + k14 * e0 * e0;
    C b1 = k13 * d1 * d1 + k14 * e1 * e1;
    C b2 = k13 * d2 * d2 + k14 * e2 * e2;
    if (sizeof(C) == 4) {
        b0 = fmin(b0, C(1e9));
        b1 = fmin(b1, C(1e9));
        b2 = fmin(b2, C(1e9));
    }
    C q0 = eps + b0, q1 = eps + b1, q2 = eps + b2;
    q0 *= q0;
    q1 *= q1;
    q2 *= q2;
    const C a0 = C(0.1) * q1 * q2, a1 = C(0.6) * q0 * q2, a2 = C(0.3) * q0 * q1;
    const C p0 = C(2) * v0 - C(7) * v1 + C(11) * v2;
    const C p1 = -v1 + C(5) * v2 + C(2) * v3;
    const C p2 = C(2) * v2 + C(5) * v3 - v4;
    return (a0 * p0 + a1 * p1 + a2 * p2) * rcp_fast(C(6) * (a0 + a1 + a2));
}

template <class Pol>
__device__ __forceinline__ typename Pol::C weno5(typename Pol::C v0, typename Pol::C v1, typename Pol::C v2,
                                                 typename Pol::C v3, typename Pol::C v4, typename Pol::C eps) {
    if constexpr (Pol::kExact) return weno5_ref(v0, v1, v2, v3, v4, eps);
    else return weno5_fast(v0, v1, v2, v3, v4, eps);
}

// ------------------------------------------------- pressure / sound speed
// EulerPhase::computePressurefromOther (EulerPhase.cpp:130-133) and
// a = sqrt(gamma p / rho) (RiemmanSolverHLL.cpp:18,24).  FP32-mixed: p and a are
// recovered in FP64 where the kinetic energy exceeds 90% of E.
template <class Pol>
__device__ __forceinline__ void finish_state(Face5<typename Pol::C>& s, double g) {
    using C = typename Pol::C;
    if constexpr (Pol::kExact) {
        s.p = (g - 1) * (s.E - 0.5 * (s.mx * s.mx + s.my * s.my) / s.r);
        s.a = sqrt(g * s.p / s.r);
    } else if constexpr (Pol::kMixed) {
        const C rinv = rcp_fast(s.r);
        s.ri = rinv;
        const C ke = C(0.5) * (s.mx * s.mx + s.my * s.my) * rinv;
        if (ke > C(0.9) * s.E) {
            const double r = s.r, mx = s.mx, my = s.my, E = s.E;
            const double p = (g - 1) * (E - 0.5 * (mx * mx + my * my) / r);
            s.p = C(p);
            s.a = C(sqrt(g * p / r));
        } else {
            s.p = C(g - 1) * (s.E - ke);
            s.a = sqrt_fast(C(g) * s.p * rinv);
        }
    } else {
        const C rinv = rcp_pos(s.r);
        s.ri = rinv;
        s.p = C(g - 1) * (s.E - C(0.5) * (s.mx * s.mx + s.my * s.my) * rinv);
        s.a = sqrt_pos(C(g) * s.p * rinv);
    }
}

// EulerMod::comFlux (EulerMod.cpp:33-54); dir 0 = X, 1 = Y.
template <class Pol>
__device__ __forceinline__ void phys_flux(const Face5<typename Pol::C>& s, int dir, typename Pol::C F[4]) {
    using C = typename Pol::C;
    if constexpr (Pol::kExact) {
        const double rho = s.r, u = s.mx, v = s.my, E = s.E, p = s.p;
        if (dir == 0) {
            F[0] = u;
            F[1] = u * u / rho + p;
            F[2] = u * v / rho;
            F[3] = (E + p) * (u / rho);
        } else {
            F[0] = v;
            F[1] = u * v / rho;
            F[2] = v * v / rho + p;
            F[3] = (E + p) * (v / rho);
        }
    } else {
        const C q = dir == 0 ? s.mx : s.my;
        const C un = q * s.ri;
        F[0] = q;
        F[1] = s.mx * un + (dir == 0 ? s.p : C(0));
        F[2] = s.my * un + (dir == 0 ? C(0) : s.p);
        F[3] = (s.E + s.p) * un;
    }
}

// RiemmanSolverHLL::Solver (RiemmanSolverHLL.cpp:5-75): PVRS star state, wave
// bounds SL = min(m_nL - aL, u* - a*L), SR = max(m_nL + aL, u* + a*R) (left
// momentum in both, as written), HLL average.  kHllDavis: bounds from the
// velocities of both sides (no reference counterpart).
template <class Pol>
__device__ __forceinline__ void hll_flux(const Face5<typename Pol::C>& L, const Face5<typename Pol::C>& R, int dir,
                                         int variant, double g, typename Pol::C F[4]) {
    using C = typename Pol::C;
    C FL[4], FR[4];
    phys_flux<Pol>(L, dir, FL);
    phys_flux<Pol>(R, dir, FR);
    const C qL = dir == 0 ? L.mx : L.my, qR = dir == 0 ? R.mx : R.my;
    const C aL = L.a, aR = R.a;
    C SL, SR;
    if constexpr (Pol::kExact) {
        const double rhoL = L.r, rhoR = R.r, pL = L.p, pR = R.p;
        if (variant == kHllReference) {
            double a_ave = 0.5 * (aL + aR);
            double rho_ave = 0.5 * (rhoL + rhoR);
            double p_star = 0.5 * (pL + pR) - 0.5 * (qR / rhoR - qL / rhoL) * rho_ave * a_ave;
            double u_star = 0.5 * (qR / rhoR + qL / rhoL) - 0.5 * (pR - pL) / (rho_ave * a_ave);
            double rho_star_L = rhoL + (qL / rhoL - u_star) * rho_ave / a_ave;
            double rho_star_R = rhoR - (qR / rhoR - u_star) * rho_ave / a_ave;
            double a_star_L = sqrt(g * p_star / rho_star_L);
            double a_star_R = sqrt(g * p_star / rho_star_R);
            SL = min_ref(qL - aL, u_star - a_star_L);
            SR = max_ref(qL + aL, u_star + a_star_R);
        } else {
            const double uL = qL / rhoL, uR = qR / rhoR;
            SL = min_ref(uL - aL, uR - aR);
            SR = max_ref(uL + aL, uR + aR);
        }
    } else {
        const C uL = qL * L.ri, uR = qR * R.ri;
        if (variant == kHllReference) {
            const C a_ave = C(0.5) * (aL + aR);
            const C rho_ave = C(0.5) * (L.r + R.r);
            const C ra = rho_ave * a_ave;
            const C inv_ra = rcp_pos(ra);  // ra > 0: mean density times mean sound speed
            const C p_star = C(0.5) * (L.p + R.p) - C(0.5) * (uR - uL) * ra;
            const C u_star = C(0.5) * (uR + uL) - C(0.5) * (R.p - L.p) * inv_ra;
            const C ratio = rho_ave * rho_ave * inv_ra;
            const C rho_star_L = L.r + (uL - u_star) * ratio;
            const C rho_star_R = R.r - (uR - u_star) * ratio;
            const C gp = C(g) * p_star;
            const C a_star_L = sqrt_fast(gp * rcp_fast(rho_star_L));
            const C a_star_R = sqrt_fast(gp * rcp_fast(rho_star_R));
            SL = min_ref(qL - aL, u_star - a_star_L);
            SR = max_ref(qL + aL, u_star + a_star_R);
        } else {
            // Davis bounds have no reference counterpart: fmin / fmax (one
            // min-max instruction each) instead of the reference's
            // compare-and-select
            SL = fmin(uL - aL, uR - aR);
            SR = fmax(uL + aL, uR + aR);
        }
    }
    if constexpr (Pol::kMixed) {
        // the HLL average on (rho, m_x) and (m_y, E) in packed FP32, then the
        // upwind cases as selects
        const float inv = rcp_fast(SR - SL);
        const float2 sr = p2(SR), msl = p2(-SL), slsr = p2(SL * SR), iv = p2(inv);
        const float2 H01 = mul2(fma2(slsr, sub2(make_float2(R.r, R.mx), make_float2(L.r, L.mx)),
                                     fma2(msl, make_float2(FR[0], FR[1]), mul2(sr, make_float2(FL[0], FL[1])))), iv);
        const float2 H23 = mul2(fma2(slsr, sub2(make_float2(R.my, R.E), make_float2(L.my, L.E)),
                                     fma2(msl, make_float2(FR[2], FR[3]), mul2(sr, make_float2(FL[2], FL[3])))), iv);
        const float H[4] = {H01.x, H01.y, H23.x, H23.y};
#pragma unroll
        for (int q = 0; q < 4; ++q) F[q] = SL >= 0 ? FL[q] : (SR <= 0 ? FR[q] : H[q]);
        return;
    } else if constexpr (!Pol::kExact) {
        // FP64 throughput form: the same shape (the average formed for every
        // face, the upwind cases selected), so no divergent branch splits the
        // face's arithmetic; where the average is selected SL < 0 < SR, so its
        // reciprocal's argument is positive (elsewhere a NaN average is
        // formed and not selected)
        const C inv = rcp_pos(SR - SL), slsr = SL * SR;
        const C dU[4] = {R.r - L.r, R.mx - L.mx, R.my - L.my, R.E - L.E};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const C H = fma(slsr, dU[q], fma(SR, FL[q], -SL * FR[q])) * inv;
            F[q] = SL >= 0 ? FL[q] : (SR <= 0 ? FR[q] : H);
        }
        return;
    }
    if (SL >= 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) F[q] = FL[q];
    } else if (SR <= 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) F[q] = FR[q];
    } else {
        const C inv_SR_SL = Pol::kExact ? C(1.0) / (SR - SL) : rcp_fast(SR - SL);
        const C dU[4] = {R.r - L.r, R.mx - L.mx, R.my - L.my, R.E - L.E};
#pragma unroll
        for (int q = 0; q < 4; ++q) F[q] = (SR * FL[q] - SL * FR[q] + SL * SR * dU[q]) * inv_SR_SL;
    }
}

// Left state from s[0..4], right state from the reversed s[5..1]
// (Weno5th::comLeftPhase / comRightPhase, Weno5th.cpp:57-81), then HLL.
template <class Pol>
__device__ __forceinline__ void face_flux(const typename Pol::C s[6][kVars], int dir, double g, typename Pol::C eps,
                                          int variant, typename Pol::C F[4]) {
    using C = typename Pol::C;
    Face5<C> L, R;
    L.r = weno5<Pol>(s[0][0], s[1][0], s[2][0], s[3][0], s[4][0], eps);
    L.mx = weno5<Pol>(s[0][1], s[1][1], s[2][1], s[3][1], s[4][1], eps);
    L.my = weno5<Pol>(s[0][2], s[1][2], s[2][2], s[3][2], s[4][2], eps);
    L.E = weno5<Pol>(s[0][3], s[1][3], s[2][3], s[3][3], s[4][3], eps);
    R.r = weno5<Pol>(s[5][0], s[4][0], s[3][0], s[2][0], s[1][0], eps);
    R.mx = weno5<Pol>(s[5][1], s[4][1], s[3][1], s[2][1], s[1][1], eps);
    R.my = weno5<Pol>(s[5][2], s[4][2], s[3][2], s[2][2], s[1][2], eps);
    R.E = weno5<Pol>(s[5][3], s[4][3], s[3][3], s[2][3], s[1][3], eps);
    finish_state<Pol>(L, g);
    finish_state<Pol>(R, g);
    hll_flux<Pol>(L, R, dir, variant, g, F);
}

// ----------------------------------------------------------- RK update
// TVD2rdRK::advance (TVD2rdRK.cpp:3-31), TVD3rdRK::advance (TVD3rdRK.cpp:3-48),
// coefficient tables TVD2rdRK.h:16-19 / TVD3rdRK.h:14-18, each product taken in
// the reference's order (coef * dt) * R.  Evaluated in FP64 for every policy.
__device__ __forceinline__ double rk_update(int rk, int stage, double dt, double cur, double u0v, double u1v, double r) {
    if (stage == 0) return 1.0 * cur + 1.0 * dt * r;
    if (rk == kRkTvd2) return 0.5 * u0v + 0.5 * cur + 0.5 * dt * r;
    if (stage == 1) return 0.75 * u0v + 0.25 * cur + 0.25 * dt * r;
    if (rk == kRkTvd3Ref) return (1.0 / 3.0) * u0v + (2.0 / 3.0) * u1v + (2.0 / 3.0) * dt * r;
    return (1.0 / 3.0) * u0v + (2.0 / 3.0) * cur + (2.0 / 3.0) * dt * r;
}

// ------------------------------------------------------ stochastic rounding
// FP32 storage of the FP32-mixed form rounds each new state value
// stochastically (no reference counterpart): to one of the two floats around
// the exact FP64 value, the farther one with probability proportional to its
// nearness.  Round-to-nearest biases the error of a smooth, slowly moving
// state (neighbouring cells and steps round the same way), so it grows with
// the step count; stochastic rounding leaves an unbiased random walk.
// Random bits: MurmurHash3's 32-bit finaliser (public domain) of a mix of cell and step.
__device__ __forceinline__ unsigned int fmix32(unsigned int h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// One finaliser over a linear mix of cell and step (odd multipliers, so
// neighbouring cells and steps enter far apart).
__device__ __forceinline__ unsigned int cell_hash(int i, int j, unsigned int step_seed) {
    return fmix32(static_cast<unsigned int>(i) * 0x9e3779b1u + static_cast<unsigned int>(j) * 0x85ebca77u +
                  step_seed * 0xc2b2ae3du);
}

// Dither of stochastic rounding for a result near f: uniform over one float
// spacing g of f's binade, (u + 1/2)/256 - 1/2 times g for the 8 random bits u
// (the low byte of `bits`), built by placing u in the mantissa of a float in
// [1, 2).  Added to a value x between neighbouring floats lo < x < lo + g
// before one round-to-nearest, it picks lo + g with probability (x - lo)/g (to
// 1/256).  Just below a power of two the spacing halves, so there the choice
// is only approximately unbiased; for |f| below 2^-103 the dither is 0 (round
// to nearest).
__device__ __forceinline__ float sr_dither(float f, unsigned int bits) {
    const int eb = static_cast<int>(__float_as_uint(f) & 0x7f800000u);
    const float g = __int_as_float(max(eb - (23 << 23), 0));
    const float m = __uint_as_float(0x3f800000u | ((bits & 255u) << 15) | (1u << 14));
    return fmaf(m, g, -1.5f * g);
}

// Positivity floors of CFS_POSITIVITY_FLOOR (no reference counterpart): a new
// state with rho <= kRhoFloor (or a NaN) becomes the floor state at rest (the
// velocity of a near-zero density is not kept: it would blow up); one with
// p <= kPFloor gets E raised so that p reaches its floor, momentum kept.
constexpr double kRhoFloor = 1e-6, kPFloor = 1e-6;
constexpr int kPosFloor = 3;

__device__ __forceinline__ void floor_state(double s[kVars], double g) {
    double rho = s[0], mx = s[1], my = s[2], E = s[3];
    if (!(rho > kRhoFloor) || !(mx == mx) || !(my == my) || !(E == E)) {
        rho = kRhoFloor;
        mx = my = 0.0;
        E = kPFloor / (g - 1);
    }
    const double ke = 0.5 * (mx * mx + my * my) / rho;
    if (!((g - 1) * (E - ke) > kPFloor)) E = kPFloor / (g - 1) + ke;
    s[0] = rho;
    s[1] = mx;
    s[2] = my;
    s[3] = E;
}

// (|u| + a)/dx + (|v| + a)/dy of one cell, FP64, in the order of the CFL
// reduction every caller shares.
__device__ __forceinline__ double wave_sum(double rho, double mx, double my, double E, double g, double dx, double dy) {
    const double p = (g - 1) * (E - 0.5 * (mx * mx + my * my) / rho);
    const double a = sqrt(g * p / rho);
    const double u = mx / rho, v = my / rho;
    return (fabs(u) + a) / dx + (fabs(v) + a) / dy;
}

// A CFL maximum takes a non-finite wave-speed sum (a NaN from a negative
// pressure or density, an infinity) as +infinity, so that one blown-up fluid
// cell makes the maximum infinite and dt = cfl / max zero, which every caller
// reports as CFS_ERR_NUMERIC (a plain `w > m` would skip NaN cells and keep
// stepping on a finite dt).
__device__ __forceinline__ double cfl_term(double w) {
    return w == w ? w : __longlong_as_double(0x7ff0000000000000LL);
}

// The same wave-speed sum for the CFL maximum fused into the last stage of the
// throughput forms: one reciprocal and one square root, in the form's
// arithmetic type (inv_dx = 1/dx, inv_dy = 1/dy).
template <class C>
__device__ __forceinline__ C wave_sum_fast(C rho, C mx, C my, C E, C g, C inv_dx, C inv_dy) {
    const C ri = rcp_fast(rho);
    const C u = mx * ri, v = my * ri;
    const C p = (g - C(1)) * (E - C(0.5) * (mx * u + my * v));
    const C a = sqrt_fast(g * p * ri);
    return (fabs(u) + a) * inv_dx + (fabs(v) + a) * inv_dy;
}

// Writes one cell of the new state and the ghost copies it feeds: Neumann
// ghosts copy the adjacent cell into all three layers (NeummanBoundary.cpp:31-45;
// one ghost repeated three times in the stencil, CellInterface.cpp:147-179),
// periodic ghosts wrap, and corner ghosts take both copies (the viscous
// stencils read them).  Dirichlet ghosts are constant and set at upload.
template <class T>
__device__ __forceinline__ void store_cell4(T* out, const Layout& L, const int bc[4], int i, int j, const T val[kVars]) {
    if (i >= kGhost && i < L.nx - kGhost && j >= kGhost && j < L.ny - kGhost) {  // no ghost copies
        st_cell<T>(out, L.offset(i, j), val);
        return;
    }
    int xi[4], yj[4];
    int nxi = 1, nyj = 1;
    xi[0] = i;
    yj[0] = j;
    if (bc[0] == kNeumann && i == 0) { xi[nxi++] = -1; xi[nxi++] = -2; xi[nxi++] = -3; }
    if (bc[1] == kNeumann && i == L.nx - 1) { xi[nxi++] = L.nx; xi[nxi++] = L.nx + 1; xi[nxi++] = L.nx + 2; }
    if (bc[0] == kPeriodic && i >= L.nx - kGhost) xi[nxi++] = i - L.nx;
    if (bc[1] == kPeriodic && i < kGhost) xi[nxi++] = i + L.nx;
    if (bc[2] == kNeumann && j == 0) { yj[nyj++] = -1; yj[nyj++] = -2; yj[nyj++] = -3; }
    if (bc[3] == kNeumann && j == L.ny - 1) { yj[nyj++] = L.ny; yj[nyj++] = L.ny + 1; yj[nyj++] = L.ny + 2; }
    if (bc[2] == kPeriodic && j >= L.ny - kGhost) yj[nyj++] = j - L.ny;
    if (bc[3] == kPeriodic && j < kGhost) yj[nyj++] = j + L.ny;
    for (int a = 0; a < nxi; ++a)
        for (int b = 0; b < nyj; ++b) st_cell<T>(out, L.offset(xi[a], yj[b]), val);
}

template <int NT>
__device__ __forceinline__ double block_max(double m, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = m;
    __syncthreads();
    if (w == 0) {
        m = (l < NT / 32) ? red[l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    return m;
}

__device__ __forceinline__ double stage_dt(const StageArgs& a) {
    if (!a.P) return a.dt;
    if (a.P->use_cfl) return a.P->cfl / __longlong_as_double(static_cast<long long>(a.P->wmax[a.parity]));
    return a.P->dt_fixed;
}

// ------------------------------------------------------------ stage kernel
// One RK stage on a TI x TJ tile: the tile and its 3-cell halo are staged in
// shared memory; every x- and y-face of the tile gets its WENO5 states and HLL
// flux (kept in shared memory, never in DRAM); each cell then forms its RHS
// (Cell::comRHS, Cell.cpp:110-126) and, if fluid, its RK update.
template <class Pol, int TI, int TJ>
__global__ void __launch_bounds__(TI * TJ) stage_kernel(const StageArgs a) {
    using T = typename Pol::T;
    using C = typename Pol::C;
    constexpr int NT = TI * TJ;
    constexpr int HI = TI + 2 * kGhost, HJ = TJ + 2 * kGhost;
    __shared__ C sU[kVars][HI][HJ];
    __shared__ C sFX[kVars][TI + 1][TJ];
    __shared__ C sFY[kVars][TI][TJ + 1];
    __shared__ double red[NT / 32];

    const Layout& L = a.L;
    const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
    const T* in = static_cast<const T*>(a.in);
    const int t = threadIdx.x;

    for (int e = t; e < HI * HJ; e += NT) {
        const int r = e / HJ, c = e - r * HJ;
        const int i = i0 - kGhost + r, j = j0 - kGhost + c;
        const bool corner = (r < kGhost || r >= TI + kGhost) && (c < kGhost || c >= TJ + kGhost);
        const bool ok = !corner && i < L.nx + kGhost && j < L.ny + kGhost;
        if (ok) {
            T cv[kVars];
            ld_cell<T>(in, L.offset(i, j), cv);
#pragma unroll
            for (int v = 0; v < kVars; ++v) sU[v][r][c] = decc<T, C>(cv[v], L, v);
        } else {
#pragma unroll
            for (int v = 0; v < kVars; ++v) sU[v][r][c] = C(0);
        }
    }
    __syncthreads();

    const C eps = C(a.eps);
    const bool lo_x = a.bc[0] == kNeumann || a.bc[0] == kDirichlet;
    const bool hi_x = a.bc[1] == kNeumann || a.bc[1] == kDirichlet;
    const bool lo_y = a.bc[2] == kNeumann || a.bc[2] == kDirichlet;
    const bool hi_y = a.bc[3] == kNeumann || a.bc[3] == kDirichlet;

    // x-normal faces: face fi (0..TI) of tile column fj lies between cells
    // i0+fi-1 and i0+fi.  On a physical boundary face the interior slots repeat
    // the first interior cell (CellInterface.cpp:172-178 stop both walkers).
    for (int f = t; f < (TI + 1) * TJ; f += NT) {
        const int fi = f / TJ, fj = f - fi * TJ;
        const int fa = i0 + fi, j = j0 + fj;
        if (fa > L.nx || j >= L.ny) continue;
        C s[6][kVars];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            int r = fi + k;
            if (fa == 0 && lo_x && k >= 3) r = fi + 3;
            if (fa == L.nx && hi_x && k <= 2) r = fi + 2;
#pragma unroll
            for (int v = 0; v < kVars; ++v) s[k][v] = sU[v][r][fj + kGhost];
        }
        C F[4];
        face_flux<Pol>(s, 0, a.gamma, eps, a.hll, F);
#pragma unroll
        for (int v = 0; v < kVars; ++v) sFX[v][fi][fj] = F[v];
    }
    // y-normal faces: face fj (0..TJ) of tile row fi between cells j0+fj-1, j0+fj.
    for (int f = t; f < TI * (TJ + 1); f += NT) {
        const int fi = f / (TJ + 1), fj = f - fi * (TJ + 1);
        const int i = i0 + fi, fb = j0 + fj;
        if (i >= L.nx || fb > L.ny) continue;
        C s[6][kVars];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            int c = fj + k;
            if (fb == 0 && lo_y && k >= 3) c = fj + 3;
            if (fb == L.ny && hi_y && k <= 2) c = fj + 2;
#pragma unroll
            for (int v = 0; v < kVars; ++v) s[k][v] = sU[v][fi + kGhost][c];
        }
        C F[4];
        face_flux<Pol>(s, 1, a.gamma, eps, a.hll, F);
#pragma unroll
        for (int v = 0; v < kVars; ++v) sFY[v][fi][fj] = F[v];
    }
    __syncthreads();

    const double dt = stage_dt(a);
    if (a.P && a.first_stage && blockIdx.x == 0 && blockIdx.y == 0 && t == 0) {
        a.P->wmax[1 - a.parity] = 0ull;
        a.P->t += dt;
        a.P->dt_last = dt;
    }

    const int ti = t / TJ, tj = t - (t / TJ) * TJ;
    const int i = i0 + ti, j = j0 + tj;
    double wloc = 0.0;
    if (i < L.nx && j < L.ny) {
        const bool fluid = a.types ? (a.types[static_cast<long long>(i) * L.ny + j] == 0) : true;
        const long long off = L.offset(i, j);
        const T* u0 = static_cast<const T*>(a.u0);
        const T* u1 = static_cast<const T*>(a.u1);
        T* out = static_cast<T*>(a.out);
        double nv[kVars];
        T sv[kVars], u0c[kVars] = {T(0), T(0), T(0), T(0)}, u1c[kVars] = {T(0), T(0), T(0), T(0)};
        if (fluid && a.stage >= 1) ld_cell<T>(u0, off, u0c);
        if (fluid && a.stage == 2 && a.rk == kRkTvd3Ref) ld_cell<T>(u1, off, u1c);
#pragma unroll
        for (int v = 0; v < kVars; ++v) {
            double rv;
            if constexpr (Pol::kExact) {
                rv = -(sFX[v][ti + 1][tj] - sFX[v][ti][tj]) / a.dx - (sFY[v][ti][tj + 1] - sFY[v][ti][tj]) / a.dy;
            } else {
                rv = -double(sFX[v][ti + 1][tj] - sFX[v][ti][tj]) / a.dx - double(sFY[v][ti][tj + 1] - sFY[v][ti][tj]) / a.dy;
            }
            if (a.rv && v >= 1)
                rv += double(static_cast<const T*>(a.rv)[static_cast<long long>(v - 1) * L.nx * L.ny + static_cast<long long>(i) * L.ny + j]);
            const double cur = double(sU[v][ti + kGhost][tj + kGhost]);
            double val = cur;
            if (fluid) {
                const double u0v = a.stage >= 1 ? dec<T>(u0c[v], L, v) : 0.0;
                const double u1v = (a.stage == 2 && a.rk == kRkTvd3Ref) ? dec<T>(u1c[v], L, v) : 0.0;
                val = rk_update(a.rk, a.stage, dt, cur, u0v, u1v, rv);
            }
            sv[v] = enc<T>(val, L, v);
            nv[v] = dec<T>(sv[v], L, v);
            if (a.rhs) a.rhs[static_cast<long long>(v) * L.nx * L.ny + static_cast<long long>(i) * L.ny + j] = fluid ? rv : 0.0;
        }
        store_cell4<T>(out, L, a.bc, i, j, sv);
        if (a.P && a.last_stage && a.P->use_cfl && fluid) {
            const double w = cfl_term(wave_sum(nv[0], nv[1], nv[2], nv[3], a.gamma, a.dx, a.dy));
            if (w > wloc) wloc = w;
        }
    }
    if (a.P && a.last_stage && a.P->use_cfl) {
        const double m = block_max<NT>(wloc, red);
        if (t == 0 && m > 0.0) atomicMax(&a.P->wmax[1 - a.parity], static_cast<unsigned long long>(__double_as_longlong(m)));
    }
}

// --------------------------------------------------- viscous (NS) terms
// No reference counterpart is live: the reference computes a viscous flux but
// never adds it (Cell.cpp:128-133, Run.cpp:177,188).  Here: u, v and
// T = gamma Ma^2 p / rho on the tile and its 3-cell halo (corners included);
// cell-centred 4th-order derivatives with the reference's table theta_c
// (FourthOrderCS.h:34-36); at each face the normal derivative from theta_r[1]
// over 6 cells (FourthOrderCS.h:28-32), the cross derivative and u, v
// interpolated with zeta_r[1] (FourthOrderCS.h:38-42); stresses
// sigma_11 = mu (4/3 u_x - 2/3 v_y), sigma_12 = mu (u_y + v_x), heat flux
// kT T_x with kT = mu / ((gamma-1) Ma^2 Pr).
// (Functions of a constant table rather than __constant__ arrays: with the
// loops unrolled every coefficient becomes an immediate, where an array read
// costs a constant-bank load and, in FP32, a conversion per use.)
__device__ __forceinline__ double theta_r1(int k) {
    constexpr double t[6] = {-3.0 / 640, 25.0 / 384, -75.0 / 64, 75.0 / 64, -25.0 / 384, 3.0 / 640};
    return t[k];
}
__device__ __forceinline__ double theta_c(int m) {
    constexpr double t[5] = {1.0 / 12, -8.0 / 12, 0.0, 8.0 / 12, -1.0 / 12};
    return t[m];
}
__device__ __forceinline__ double zeta1(int k) {
    constexpr double t[4] = {-1.0 / 16, 9.0 / 16, 9.0 / 16, -1.0 / 16};
    return t[k];
}

template <class Pol, int TI, int TJ>
__global__ void __launch_bounds__(TI * TJ) viscous_kernel(const ViscArgs a) {
    using T = typename Pol::T;
    using C = typename Pol::C;
    constexpr int HI = TI + 2 * kGhost, HJ = TJ + 2 * kGhost;
    __shared__ C sP[3][HI][HJ];
    __shared__ C sGY[3][TI + 4][TJ];
    __shared__ C sGX[3][TI][TJ + 4];
    __shared__ C sFV[3][TI + 1][TJ];
    __shared__ C sGV[3][TI][TJ + 1];
    const Layout& L = a.L;
    const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
    const T* in = static_cast<const T*>(a.in);
    const int t = threadIdx.x;
    constexpr bool kF = sizeof(C) == 4;  // FP32 form: constants rounded on the host
    const C gm1 = kF ? C(a.gm1_f) : C(a.gamma - 1), cT = kF ? C(a.cT_f) : C(a.gamma * a.mach2);
    // threads as a TI x TJ grid (TJ = 32: one warp per row).  Phases walk rows
    // by warp and columns by lane.  Items past column TJ (TJ + 4 x-derivatives
    // and TJ + 1 y-normal faces per row) go to one short extra pass whose lanes
    // lie whole tile rows apart (distinct shared-memory banks); x-derivatives
    // and x-normal faces take two rows per thread; the halo tile (TJ + 6 per
    // row, stored only) numbers its cells row by row over all threads.  So no
    // warp makes a second pass for a few items.
    static_assert(TJ == 32, "one warp per tile row");
    constexpr int NT = TI * TJ;
    const int ty = t / TJ, tx = t - ty * TJ;
    for (int e = t; e < HI * HJ; e += NT) {
        const int r = e / HJ, c = e - r * HJ;
        const int i = i0 - kGhost + r, j = j0 - kGhost + c;
        C u = C(0), v = C(0), Tt = C(0);
        if (i < L.nx + kGhost && j < L.ny + kGhost) {
            T cv[kVars];
            ld_cell<T>(in, L.offset(i, j), cv);
            const C rho = decc<T, C>(cv[0], L, 0), mx = decc<T, C>(cv[1], L, 1);
            const C my = decc<T, C>(cv[2], L, 2), E = decc<T, C>(cv[3], L, 3);
            const C rinv = rcp_fast(rho);
            u = mx * rinv;
            v = my * rinv;
            const C p = gm1 * (E - C(0.5) * (mx * mx + my * my) * rinv);
            Tt = cT * p * rinv;
        }
        sP[0][r][c] = u;
        sP[1][r][c] = v;
        sP[2][r][c] = Tt;
    }
    __syncthreads();
    const C idx = kF ? C(a.inv_dx_f) : C(a.inv_dx), idy = kF ? C(a.inv_dy_f) : C(a.inv_dy);
    for (int rr = ty; rr < TI + 4; rr += TI) {  // y-derivatives of rows i0-2 .. i0+TI+1
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            C s = C(0);
#pragma unroll
            for (int m = 0; m < 5; ++m) s += C(theta_c(m)) * sP[q][rr + 1][tx + 1 + m];
            sGY[q][rr][tx] = s * idy;
        }
    }
    // x-derivatives of columns j0-2 .. j0+TJ+1, rows rr and rr+1 per thread
    // (four of their five stencil values shared): columns 0..TJ-1 by lane,
    // the 4 past them in a tail whose lanes lie two tile rows apart; on the
    // top warps, as the y-derivatives' second pass runs on the bottom ones
    static_assert(TI % 2 == 0, "row pairs");
    {
        constexpr int kMain = (TI / 2) * TJ, kCount = kMain + 4 * (TI / 2);
        constexpr int kFirst = NT - (kCount + 31) / 32 * 32;
        static_assert(kFirst >= 0, "x-derivative pairs fit in one pass");
        const int u = t - kFirst;
        if (u >= 0 && u < kCount) {
            const int pr = u < kMain ? u / TJ : (u - kMain) % (TI / 2);
            const int cc = u < kMain ? u % TJ : TJ + (u - kMain) / (TI / 2);
            const int rr = 2 * pr;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                C col[6];
#pragma unroll
                for (int m = 0; m < 6; ++m) col[m] = sP[q][rr + 1 + m][cc + 1];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    C s = C(0);
#pragma unroll
                    for (int m = 0; m < 5; ++m) s += C(theta_c(m)) * col[h + m];
                    sGX[q][rr + h][cc] = s * idx;
                }
            }
        }
    }
    __syncthreads();
    const C mu = kF ? C(a.mu_f) : C(a.mu), kT = kF ? C(a.kT_f) : C(a.kT), c43 = C(4.0 / 3.0), c23 = C(2.0 / 3.0);
    // x-normal faces between rows i0+fi-1 and i0+fi, faces fi0 and fi0+1 of a
    // column per thread (five of their six stencil values shared; TI + 1
    // faces per column, so the last pair has one face); on the top warps, as
    // the y-normal faces' tail runs on the bottom one
    {
        constexpr int kCount = (TI + 2) / 2 * TJ;
        constexpr int kFirst = NT - kCount;
        static_assert(kFirst >= 0, "x-face pairs fit in one pass");
        const int u = t - kFirst;
        if (u >= 0) {
            const int fi0 = 2 * (u / TJ), fj = u % TJ;
            const bool two = fi0 + 1 <= TI;
            C dn[2][3], cr[2][3], uf[2] = {C(0), C(0)}, vf[2] = {C(0), C(0)};
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                C col[7], gy[5];
#pragma unroll
                for (int k = 0; k < 6; ++k) col[k] = sP[q][fi0 + k][fj + kGhost];
#pragma unroll
                for (int k = 0; k < 4; ++k) gy[k] = sGY[q][fi0 + k][fj];
                col[6] = C(0);
                gy[4] = C(0);
                if (two) {
                    col[6] = sP[q][fi0 + 6][fj + kGhost];
                    gy[4] = sGY[q][fi0 + 4][fj];
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    C s = C(0), x = C(0);
#pragma unroll
                    for (int k = 0; k < 6; ++k) s += C(theta_r1(k)) * col[h + k];
#pragma unroll
                    for (int k = 0; k < 4; ++k) x += C(zeta1(k)) * gy[h + k];
                    dn[h][q] = s * idx;
                    cr[h][q] = x;
                    if (q < 2) {
                        C w = C(0);
#pragma unroll
                        for (int k = 0; k < 4; ++k) w += C(zeta1(k)) * col[h + 1 + k];
                        if (q == 0) uf[h] = w;
                        else vf[h] = w;
                    }
                }
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (h == 1 && !two) break;
                const int fi = fi0 + h;
                const C s11 = mu * (c43 * dn[h][0] - c23 * cr[h][1]);
                const C s12 = mu * (cr[h][0] + dn[h][1]);
                sFV[0][fi][fj] = s11;
                sFV[1][fi][fj] = s12;
                sFV[2][fi][fj] = uf[h] * s11 + vf[h] * s12 + kT * dn[h][2];
            }
        }
    }
    for (int pass = 0; pass < 2; ++pass) {  // y-normal faces between columns j0+fj-1 and j0+fj
        if (pass == 1 && t >= TI) break;
        const int fi = pass == 0 ? ty : t, fj = pass == 0 ? tx : TJ;
        C dn[3], cr[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            C s = C(0), x = C(0);
#pragma unroll
            for (int k = 0; k < 6; ++k) s += C(theta_r1(k)) * sP[q][fi + kGhost][fj + k];
#pragma unroll
            for (int k = 0; k < 4; ++k) x += C(zeta1(k)) * sGX[q][fi][fj + k];
            dn[q] = s * idy;
            cr[q] = x;
        }
        C uf = C(0), vf = C(0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uf += C(zeta1(k)) * sP[0][fi + kGhost][fj + 1 + k];
            vf += C(zeta1(k)) * sP[1][fi + kGhost][fj + 1 + k];
        }
        const C s22 = mu * (c43 * dn[1] - c23 * cr[0]);
        const C s21 = mu * (dn[0] + cr[1]);
        sGV[0][fi][fj] = s21;
        sGV[1][fi][fj] = s22;
        sGV[2][fi][fj] = uf * s21 + vf * s22 + kT * dn[2];
    }
    __syncthreads();
    const int ti = t / TJ, tj = t - (t / TJ) * TJ;
    const int i = i0 + ti, j = j0 + tj;
    if (i < L.nx && j < L.ny) {
        T* rv = static_cast<T*>(a.rv);
        const long long n = static_cast<long long>(L.nx) * L.ny, k = static_cast<long long>(i) * L.ny + j;
#pragma unroll
        for (int q = 0; q < 3; ++q)
            rv[q * n + k] = T((sFV[q][ti + 1][tj] - sFV[q][ti][tj]) * idx + (sGV[q][ti][tj + 1] - sGV[q][ti][tj]) * idy);
    }
}

// -------------------------------------------------- immersed-ghost fill
// Cell::comImmersedGhostPhase -> ImagePoint::InterpolatePhase
// (Cell.cpp:172-181, ImagePoint.cpp:20-82).  Mode 0 replays the solve of the
// donor matrix's pivoted LDL^T (factor computed once on the host from the
// lower triangle, as Eigen's ldlt() reads it): permute, unit-lower forward
// substitution, pseudo-inverse of D, back substitution, un-permute; then
// W0 X Y + W1 X + W2 Y + W3 and both momenta negated.  Mode 1: bilinear
// weights and reflection of the wall-normal momentum only.  FP64 arithmetic.
template <class T>
__device__ __forceinline__ void ib_fill_one(const IbArgs& a, int g) {
    const Layout& L = a.L;
    T* U = static_cast<T*>(a.U);
    double f[kVars][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int d = a.donor[4 * g + k];
        const int i = d / L.ny, j = d - (d / L.ny) * L.ny;
        T cv[kVars];
        ld_cell<T>(U, L.offset(i, j), cv);
#pragma unroll
        for (int v = 0; v < kVars; ++v) f[v][k] = dec<T>(cv[v], L, v);
    }
    const double* fac = a.fac + 16 * g;
    double val[kVars];
    if (a.mode == 0) {
        const double X = a.image[2 * g], Y = a.image[2 * g + 1];
        const double l10 = fac[0], l20 = fac[1], l21 = fac[2], l30 = fac[3], l31 = fac[4], l32 = fac[5];
        const double dd[4] = {fac[6], fac[7], fac[8], fac[9]};
        const int* pm = a.perm + 4 * g;
#pragma unroll
        for (int v = 0; v < kVars; ++v) {
            double y[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) y[k] = f[v][pm[k]];
            y[1] -= l10 * y[0];
            y[2] -= l20 * y[0];
            y[2] -= l21 * y[1];
            y[3] -= l30 * y[0];
            y[3] -= l31 * y[1];
            y[3] -= l32 * y[2];
#pragma unroll
            for (int k = 0; k < 4; ++k) y[k] = (fabs(dd[k]) > DBL_MIN) ? y[k] / dd[k] : 0.0;
            y[2] -= l32 * y[3];
            y[1] -= l21 * y[2];
            y[1] -= l31 * y[3];
            y[0] -= l10 * y[1];
            y[0] -= l20 * y[2];
            y[0] -= l30 * y[3];
            double W[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) W[pm[k]] = y[k];
            val[v] = W[0] * X * Y + W[1] * X + W[2] * Y + W[3];
        }
        val[1] = -val[1];
        val[2] = -val[2];
    } else {
#pragma unroll
        for (int v = 0; v < kVars; ++v) val[v] = fac[0] * f[v][0] + fac[1] * f[v][1] + fac[2] * f[v][2] + fac[3] * f[v][3];
        const double nx_ = fac[4], ny_ = fac[5];
        const double mn = val[1] * nx_ + val[2] * ny_;
        val[1] = val[1] - 2.0 * mn * nx_;
        val[2] = val[2] - 2.0 * mn * ny_;
    }
    const int c = a.cell[g];
    T sv[kVars];
#pragma unroll
    for (int v = 0; v < kVars; ++v) sv[v] = enc<T>(val[v], L, v);
    st_cell<T>(U, L.offset(c / L.ny, c - (c / L.ny) * L.ny), sv);
}

template <class T>
__global__ void ib_fill_kernel(const IbArgs a) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.n) return;
    ib_fill_one<T>(a, g);
}

// Batched form: immersed-ghost cell g of the batch is cell local[g] of case
// cases[g]; args[c] is case c's fill description (its state buffer, layout, lists).
template <class T>
__global__ void batch_ib_fill_kernel(const IbArgs* __restrict__ args, const int* __restrict__ cases,
                                     const int* __restrict__ local, int total) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const IbArgs a = args[cases[g]];
    ib_fill_one<T>(a, local[g]);
}

// ------------------------------------------------------ CFL reduction
template <class T, int NT>
__global__ void __launch_bounds__(NT) wmax_kernel(const T* U, const Layout L, const uint8_t* types, double g,
                                                  double dx, double dy, unsigned long long* out) {
    __shared__ double red[NT / 32];
    double m = 0.0;
    const long long n = static_cast<long long>(L.nx) * L.ny;
    for (long long k = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; k < n; k += static_cast<long long>(gridDim.x) * NT) {
        if (types && types[k] != 0) continue;
        const int i = static_cast<int>(k / L.ny), j = static_cast<int>(k - (k / L.ny) * L.ny);
        T cv[kVars];
        ld_cell<T>(U, L.offset(i, j), cv);
        const double w = cfl_term(wave_sum(dec<T>(cv[0], L, 0), dec<T>(cv[1], L, 1), dec<T>(cv[2], L, 2),
                                           dec<T>(cv[3], L, 3), g, dx, dy));
        if (w > m) m = w;
    }
    m = block_max<NT>(m, red);
    if (threadIdx.x == 0 && m > 0.0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(m)));
}

// Batched form: blockIdx.y = case; the state is args[c].in, the maximum goes
// to args[c].P->wmax[0].
template <class T, int NT>
__global__ void __launch_bounds__(NT) batch_wmax_kernel(const StageArgs* __restrict__ args) {
    __shared__ double red[NT / 32];
    const StageArgs& a = args[blockIdx.y];
    const T* U = static_cast<const T*>(a.in);
    const Layout& L = a.L;
    double m = 0.0;
    const long long n = static_cast<long long>(L.nx) * L.ny;
    for (long long k = blockIdx.x * static_cast<long long>(NT) + threadIdx.x; k < n; k += static_cast<long long>(gridDim.x) * NT) {
        if (a.types && a.types[k] != 0) continue;
        const int i = static_cast<int>(k / L.ny), j = static_cast<int>(k - (k / L.ny) * L.ny);
        T cv[kVars];
        ld_cell<T>(U, L.offset(i, j), cv);
        const double w = cfl_term(wave_sum(dec<T>(cv[0], L, 0), dec<T>(cv[1], L, 1), dec<T>(cv[2], L, 2),
                                           dec<T>(cv[3], L, 3), a.gamma, a.dx, a.dy));
        if (w > m) m = w;
    }
    m = block_max<NT>(m, red);
    if (threadIdx.x == 0 && m > 0.0) atomicMax(&a.P->wmax[0], static_cast<unsigned long long>(__double_as_longlong(m)));
}

// Sums of rho, m_x, m_y, E over fluid cells (FP64 accumulation), in a fixed
// order so that the totals are the same bits on every run: block b of plane
// blockIdx.y sums the cells b, b + NB*NT, ... of each of its threads, reduces
// them as a tree, and writes partial[v * NB + b]; plane_final_sums_kernel adds
// the partials in index order.
template <class T, int NT, int NB>
__global__ void __launch_bounds__(NT) totals_partial_kernel(const T* U, const Layout L, const uint8_t* types,
                                                            double* partial) {
    __shared__ double red[NT];
    const int v = blockIdx.y;
    const long long n = static_cast<long long>(L.nx) * L.ny;
    double s = 0.0;
    for (long long k = static_cast<long long>(blockIdx.x) * NT + threadIdx.x; k < n; k += static_cast<long long>(NB) * NT) {
        if (types && types[k] != 0) continue;
        const int i = static_cast<int>(k / L.ny), j = static_cast<int>(k - (k / L.ny) * L.ny);
        s += dec<T>(U[Layout::at(L.offset(i, j), v)], L, v);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = NT / 2; w > 0; w >>= 1) {
        if (static_cast<int>(threadIdx.x) < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[v * NB + blockIdx.x] = red[0];
}

// --------------------------------------------- layout conversion / ghosts
// Host order [4][nx][ny] doubles <-> padded device planes.
template <class T>
__global__ void pack_kernel(const double* src, T* dst, const Layout L) {
    const long long n = static_cast<long long>(L.nx) * L.ny;
    for (long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; k < kVars * n;
         k += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int v = static_cast<int>(k / n);
        const long long c = k - v * n;
        const int i = static_cast<int>(c / L.ny), j = static_cast<int>(c - (c / L.ny) * L.ny);
        dst[Layout::at(L.offset(i, j), v)] = enc<T>(src[k], L, v);
    }
}

template <class T>
__global__ void unpack_kernel(const T* src, double* dst, const Layout L) {
    const long long n = static_cast<long long>(L.nx) * L.ny;
    for (long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; k < kVars * n;
         k += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int v = static_cast<int>(k / n);
        const long long c = k - v * n;
        const int i = static_cast<int>(c / L.ny), j = static_cast<int>(c - (c / L.ny) * L.ny);
        dst[k] = dec<T>(src[Layout::at(L.offset(i, j), v)], L, v);
    }
}

// Fills all ghost layers of a state from its interior: Neumann copies of the
// adjacent cell, periodic wraps, Dirichlet constants (conserved), as
// CartesianMesh::ApplyBoundaryCondition does once before the loop (Run.cpp:128).
// Corner ghosts apply the x side's rule first, then the y side's.
template <class T>
__device__ __forceinline__ bool ghost_value(const T* p, const Layout& L, const BcSides& sides, int v, int gi, int gj,
                                            T& out) {
    int i = gi, j = gj;
    if (gi < 0 || gi >= L.nx) {
        const int s = gi < 0 ? 0 : 1;
        const int bc = sides.bc[s];
        if (bc == kDirichlet) { out = enc<T>(sides.U[s][v], L, v); return true; }
        if (bc == kNeumann) i = gi < 0 ? 0 : L.nx - 1;
        else if (bc == kPeriodic) i = gi < 0 ? gi + L.nx : gi - L.nx;
        else return false;
    }
    if (gj < 0 || gj >= L.ny) {
        const int s = gj < 0 ? 2 : 3;
        const int bc = sides.bc[s];
        if (bc == kDirichlet) { out = enc<T>(sides.U[s][v], L, v); return true; }
        if (bc == kNeumann) j = gj < 0 ? 0 : L.ny - 1;
        else if (bc == kPeriodic) j = gj < 0 ? gj + L.ny : gj - L.ny;
        else return false;
    }
    out = p[Layout::at(L.offset(i, j), v)];
    return true;
}

template <class T>
__global__ void ghost_fill_kernel(T* U, const Layout L, BcSides sides) {
    const int per = (L.nx > L.ny ? L.nx : L.ny);
    const long long edge_items = 4LL * kGhost * per * kVars;
    const long long corner_items = 4LL * kGhost * kGhost * kVars;
    for (long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; k < edge_items + corner_items;
         k += static_cast<long long>(gridDim.x) * blockDim.x) {
        int gi, gj, v;
        if (k < edge_items) {
            v = static_cast<int>(k % kVars);
            long long rest = k / kVars;
            const int pos = static_cast<int>(rest % per);
            rest /= per;
            const int layer = static_cast<int>(rest % kGhost) + 1;
            const int side = static_cast<int>(rest / kGhost);
            if (side < 2) {
                if (pos >= L.ny) continue;
                gi = side == 0 ? -layer : L.nx - 1 + layer;
                gj = pos;
            } else {
                if (pos >= L.nx) continue;
                gi = pos;
                gj = side == 2 ? -layer : L.ny - 1 + layer;
            }
        } else {
            long long c = k - edge_items;
            v = static_cast<int>(c % kVars);
            c /= kVars;
            const int ly = static_cast<int>(c % kGhost) + 1;
            c /= kGhost;
            const int lx = static_cast<int>(c % kGhost) + 1;
            const int corner = static_cast<int>(c / kGhost);
            gi = (corner & 1) ? L.nx - 1 + lx : -lx;
            gj = (corner & 2) ? L.ny - 1 + ly : -ly;
        }
        T val;
        if (ghost_value<T>(U, L, sides, v, gi, gj, val)) U[Layout::at(L.offset(gi, gj), v)] = val;
    }
}

// ------------------------------------------------- unit-level batches
template <class Pol>
__global__ void weno_faces_kernel(int n, const double* st, double* left, double* right, double g, double eps) {
    using C = typename Pol::C;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    C s[6][kVars];
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
        for (int v = 0; v < kVars; ++v) s[k][v] = C(st[(f * 6 + k) * kVars + v]);
    Face5<C> L, R;
    const C e = C(eps);
    L.r = weno5<Pol>(s[0][0], s[1][0], s[2][0], s[3][0], s[4][0], e);
    L.mx = weno5<Pol>(s[0][1], s[1][1], s[2][1], s[3][1], s[4][1], e);
    L.my = weno5<Pol>(s[0][2], s[1][2], s[2][2], s[3][2], s[4][2], e);
    L.E = weno5<Pol>(s[0][3], s[1][3], s[2][3], s[3][3], s[4][3], e);
    R.r = weno5<Pol>(s[5][0], s[4][0], s[3][0], s[2][0], s[1][0], e);
    R.mx = weno5<Pol>(s[5][1], s[4][1], s[3][1], s[2][1], s[1][1], e);
    R.my = weno5<Pol>(s[5][2], s[4][2], s[3][2], s[2][2], s[1][2], e);
    R.E = weno5<Pol>(s[5][3], s[4][3], s[3][3], s[2][3], s[1][3], e);
    finish_state<Pol>(L, g);
    finish_state<Pol>(R, g);
    const Face5<C>* st2[2] = {&L, &R};
    double* o[2] = {left + 5 * f, right + 5 * f};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        o[q][0] = st2[q]->r;
        o[q][1] = st2[q]->mx;
        o[q][2] = st2[q]->my;
        o[q][3] = st2[q]->E;
        o[q][4] = st2[q]->p;
    }
}

template <class Pol>
__global__ void hll_faces_kernel(int n, int dir, const double* Lh, const double* Rh, double* F, double g, int variant) {
    using C = typename Pol::C;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    Face5<C> L, R;
    L.r = C(Lh[4 * f]); L.mx = C(Lh[4 * f + 1]); L.my = C(Lh[4 * f + 2]); L.E = C(Lh[4 * f + 3]);
    R.r = C(Rh[4 * f]); R.mx = C(Rh[4 * f + 1]); R.my = C(Rh[4 * f + 2]); R.E = C(Rh[4 * f + 3]);
    finish_state<Pol>(L, g);
    finish_state<Pol>(R, g);
    C out[4];
    hll_flux<Pol>(L, R, dir, variant, g, out);
#pragma unroll
    for (int q = 0; q < 4; ++q) F[4 * f + q] = out[q];
}

}  // namespace cfs
