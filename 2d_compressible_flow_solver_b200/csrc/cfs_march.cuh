// Row-marching stage kernel of the throughput forms (CFS_FP64, CFS_FP32_MIXED).
//
// Work decomposition: a warp owns a segment of kSeg = 30 consecutive y-cells
// (columns j0 .. j0+29); its 32 lanes hold columns j0-1 .. j0+30, so every
// interior cell has both y-neighbours' reconstructions inside the warp.  The
// warp marches down x (rows) from i0-1 to i1:
//  * the x-stencil of a lane is a 5-row register window of its column, one new
//    row loaded per step (no shared memory, no block barrier);
//  * the y-stencil comes from a per-warp row buffer in shared memory (the 32
//    lane values plus 2 halo columns each side), synchronised with __syncwarp;
//  * each cell reconstructs its own left- and right-biased WENO5 states per
//    direction and variable from ONE set of smoothness indicators (the
//    indicators of the two states are the same three numbers in mirrored
//    order), then each face's HLL flux takes the left state of the cell below
//    it and the right state of the cell above (a shuffle in y, the previous
//    march step in x);
//  * the RK update of row r-1 happens at step r, when its upper x-face exists.
// Physical boundary faces use the reference's stencil (CellInterface.cpp:
// 172-178: both walkers stop, so interior slots repeat the first interior cell).
#pragma once
#include "cfs_kernels.cuh"

namespace cfs {

constexpr int kSeg = 30;

// Left- and right-biased WENO5 states of the middle cell of v0..v4
// (Weno5th.cpp:4-28 applied to v0..v4 and to v4..v0), rewritten on the
// differences D1..D4 (Dk = v_k - v_{k-1}) so that both states share one set of
// smoothness indicators and weight products and are formed as v2 plus a small
// correction (fewer operations, and in FP32 a rounding error relative to the
// correction instead of to the value):
//   beta_k (13/12) d_k^2 + (1/4) e_k^2 with d = (D2-D1, D3-D2, D4-D3),
//     e = (3 D2 - D1, D2 + D3, D4 - 3 D3) = (2 D2 + d0, D2 + D3, D4 - 3 D3);
//     scaled by 12/13 with eps alike, which leaves the normalised weights
//     unchanged;
//   candidate p_k = v2 + c_k: c = ((5 D2 - 2 D1)/6, (D2 + 2 D3)/6, (4 D3 - D4)/6),
//     mirrored c' = ((2 D4 - 5 D3)/6, -(D3 + 2 D2)/6, (D1 - 4 D2)/6); each
//     mirrored candidate is d/6 minus a left one: c'_0 = d2/6 - c_2,
//     c'_1 = d1/6 - c_1, c'_2 = d0/6 - c_0, so the left ones are formed
//     negated (n_k = -c_k) and the right ones take one fused multiply-add;
//   weights d_k / q_k with q_k = (eps + beta_k)^2, taken as products of the
//     other two q times (1, 6, 3) (the linear weights 0.1, 0.6, 0.3 times 10).
template <class C>
__device__ __forceinline__ void weno5_pair_diff(C v0, C v1, C v2, C v3, C v4, C eps, C& left, C& right) {
    const C D1 = v1 - v0, D2 = v2 - v1, D3 = v3 - v2, D4 = v4 - v3;
    const C d0 = D2 - D1, d1 = D3 - D2, d2 = D4 - D3;
    const C e0 = fma(C(2), D2, d0), e1 = D2 + D3, e2 = fma(C(-3), D3, D4);
    const C k = C(3.0 / 13.0);
    C b0 = fma(d0, d0, k * (e0 * e0));
    C b1 = fma(d1, d1, k * (e1 * e1));
    C b2 = fma(d2, d2, k * (e2 * e2));
    if (sizeof(C) == 4) {
        b0 = fmin(b0, C(1e9));
        b1 = fmin(b1, C(1e9));
        b2 = fmin(b2, C(1e9));
    }
    C q0 = eps + b0, q1 = eps + b1, q2 = eps + b2;  // eps: the WENO eps times 12/13
    q0 *= q0;
    q1 *= q1;
    q2 *= q2;
    const C q01 = q0 * q1, q12 = q1 * q2, a1 = C(6) * (q0 * q2);
    const C a2L = C(3) * q01, a2R = C(3) * q12;
    const C n0 = fma(C(-5.0 / 6.0), D2, C(1.0 / 3.0) * D1);
    const C n1 = fma(C(-1.0 / 3.0), D3, C(-1.0 / 6.0) * D2);
    const C n2 = fma(C(-2.0 / 3.0), D3, C(1.0 / 6.0) * D4);
    const C r0 = fma(C(1.0 / 6.0), d2, n2);
    const C r1 = fma(C(1.0 / 6.0), d1, n1);
    const C r2 = fma(C(1.0 / 6.0), d0, n0);
    // (the weight sums are >= eps^2 > 0: rcp_pos; the left one negated after)
    left = fma(fma(q12, n0, fma(a1, n1, a2L * n2)), -rcp_pos(q12 + a1 + a2L), v2);
    right = fma(fma(q01, r0, fma(a1, r1, a2R * r2)), rcp_pos(q01 + a1 + a2R), v2);
}

template <class C>
__device__ __forceinline__ void weno5_pair(C v0, C v1, C v2, C v3, C v4, C eps, C& left, C& right) {
    weno5_pair_diff(v0, v1, v2, v3, v4, C(12.0 / 13.0) * eps, left, right);
}

// The same pair for two variables at once in packed FP32 (sm_100 FFMA2 /
// FADD2 / FMUL2: two independent FP32 operations per instruction, each rounded
// as its scalar form), for the FP32-mixed form, whose row loop is bound by
// instruction issue.  The reciprocals stay scalar.

__device__ __forceinline__ void weno5_pair_x2(float2 v0, float2 v1, float2 v2, float2 v3, float2 v4, float eps,
                                              float2& left, float2& right) {
    const float2 D1 = sub2(v1, v0), D2 = sub2(v2, v1), D3 = sub2(v3, v2), D4 = sub2(v4, v3);
    const float2 d0 = sub2(D2, D1), d1 = sub2(D3, D2), d2 = sub2(D4, D3);
    const float2 e0 = fma2(p2(2.0f), D2, d0), e1 = add2(D2, D3), e2 = fma2(p2(-3.0f), D3, D4);
    const float2 k = p2(float(3.0 / 13.0));
    float2 b0 = fma2(d0, d0, mul2(k, mul2(e0, e0)));
    float2 b1 = fma2(d1, d1, mul2(k, mul2(e1, e1)));
    float2 b2 = fma2(d2, d2, mul2(k, mul2(e2, e2)));
    b0 = make_float2(fminf(b0.x, 1e9f), fminf(b0.y, 1e9f));
    b1 = make_float2(fminf(b1.x, 1e9f), fminf(b1.y, 1e9f));
    b2 = make_float2(fminf(b2.x, 1e9f), fminf(b2.y, 1e9f));
    const float2 es = p2(float(12.0 / 13.0) * eps);
    float2 q0 = add2(es, b0), q1 = add2(es, b1), q2 = add2(es, b2);
    q0 = mul2(q0, q0);
    q1 = mul2(q1, q1);
    q2 = mul2(q2, q2);
    const float2 q01 = mul2(q0, q1), q12 = mul2(q1, q2), a1 = mul2(p2(6.0f), mul2(q0, q2));
    const float2 a2L = mul2(p2(3.0f), q01), a2R = mul2(p2(3.0f), q12);
    const float2 n0 = fma2(p2(float(-5.0 / 6.0)), D2, mul2(p2(float(1.0 / 3.0)), D1));
    const float2 n1 = fma2(p2(float(-1.0 / 3.0)), D3, mul2(p2(float(-1.0 / 6.0)), D2));
    const float2 n2 = fma2(p2(float(-2.0 / 3.0)), D3, mul2(p2(float(1.0 / 6.0)), D4));
    const float2 sixth = p2(float(1.0 / 6.0));
    const float2 r0 = fma2(sixth, d2, n2), r1 = fma2(sixth, d1, n1), r2 = fma2(sixth, d0, n0);
    const float2 sL = add2(add2(q12, a1), a2L), sR = add2(add2(q01, a1), a2R);
    // (the left reciprocals negated: the left sum is over the negated candidates)
    const float2 iL = make_float2(rcp_fast(-sL.x), rcp_fast(-sL.y)), iR = make_float2(rcp_fast(sR.x), rcp_fast(sR.y));
    left = fma2(fma2(q12, n0, fma2(a1, n1, mul2(a2L, n2))), iL, v2);
    right = fma2(fma2(q01, r0, fma2(a1, r1, mul2(a2R, r2))), iR, v2);
}

// finish_state of a cell's two states at once (FP32-mixed: packed
// instructions; a state whose kinetic energy exceeds 90 % of E takes the scalar
// path with its FP64 pressure).
template <class Pol>
__device__ __forceinline__ void finish_pair(Face5<typename Pol::C>& L, Face5<typename Pol::C>& R, double g) {
    if constexpr (Pol::kMixed) {
        const float2 mx = make_float2(L.mx, R.mx), my = make_float2(L.my, R.my), E = make_float2(L.E, R.E);
        const float2 ri = make_float2(rcp_fast(L.r), rcp_fast(R.r));
        const float2 ke = mul2(mul2(p2(0.5f), fma2(mx, mx, mul2(my, my))), ri);
        if (ke.x > 0.9f * L.E || ke.y > 0.9f * R.E) {
            finish_state<Pol>(L, g);
            finish_state<Pol>(R, g);
            return;
        }
        const float2 p = mul2(p2(float(g - 1)), sub2(E, ke));
        const float2 a2 = mul2(mul2(p2(float(g)), p), ri);
        const float2 a = mul2(a2, make_float2(rsqrt_fast(a2.x), rsqrt_fast(a2.y)));
        L.ri = ri.x;
        R.ri = ri.y;
        L.p = p.x;
        R.p = p.y;
        L.a = a.x;
        R.a = a.y;
    } else {
        finish_state<Pol>(L, g);
        finish_state<Pol>(R, g);
    }
}

// Both states of one cell from a 5-cell stencil st[k][v] (k = 0..4).  The
// FP32-mixed form pairs (rho, rho u) and (rho v, E) in packed instructions.
// With `off` the stencil holds stored deviations (value - off[v]): WENO5 is
// translation invariant (the difference form sees only differences), so the
// states are reconstructed from the deviations and the offsets added once.
template <class Pol>
__device__ __forceinline__ void cell_states(const typename Pol::C st[5][kVars], typename Pol::C eps, double g,
                                            Face5<typename Pol::C>& L, Face5<typename Pol::C>& R,
                                            const float* off = nullptr) {
    if constexpr (Pol::kMixed) {
        float2 l, r;
        weno5_pair_x2(make_float2(st[0][0], st[0][1]), make_float2(st[1][0], st[1][1]), make_float2(st[2][0], st[2][1]),
                      make_float2(st[3][0], st[3][1]), make_float2(st[4][0], st[4][1]), eps, l, r);
        if (off) {
            const float2 o = make_float2(off[0], off[1]);
            l = add2(l, o);
            r = add2(r, o);
        }
        L.r = l.x;
        L.mx = l.y;
        R.r = r.x;
        R.mx = r.y;
        weno5_pair_x2(make_float2(st[0][2], st[0][3]), make_float2(st[1][2], st[1][3]), make_float2(st[2][2], st[2][3]),
                      make_float2(st[3][2], st[3][3]), make_float2(st[4][2], st[4][3]), eps, l, r);
        if (off) {
            const float2 o = make_float2(off[2], off[3]);
            l = add2(l, o);
            r = add2(r, o);
        }
        L.my = l.x;
        L.E = l.y;
        R.my = r.x;
        R.E = r.y;
    } else {
        weno5_pair(st[0][0], st[1][0], st[2][0], st[3][0], st[4][0], eps, L.r, R.r);
        weno5_pair(st[0][1], st[1][1], st[2][1], st[3][1], st[4][1], eps, L.mx, R.mx);
        weno5_pair(st[0][2], st[1][2], st[2][2], st[3][2], st[4][2], eps, L.my, R.my);
        weno5_pair(st[0][3], st[1][3], st[2][3], st[3][3], st[4][3], eps, L.E, R.E);
    }
    finish_pair<Pol>(L, R, g);
}

// Reference boundary face between an interior cell value c and a ghost value g
// (lo = true: ghost below, stencil [g g g | c c c]; lo = false: [c c c | g g g]).
template <class Pol>
__device__ __forceinline__ void boundary_face_states(const typename Pol::C c[kVars], const typename Pol::C gh[kVars],
                                                     bool lo, typename Pol::C eps, double g,
                                                     Face5<typename Pol::C>& L, Face5<typename Pol::C>& R) {
    using C = typename Pol::C;
    C* lp[4] = {&L.r, &L.mx, &L.my, &L.E};
    C* rp[4] = {&R.r, &R.mx, &R.my, &R.E};
#pragma unroll
    for (int v = 0; v < kVars; ++v) {
        const C a = lo ? gh[v] : c[v], b = lo ? c[v] : gh[v];
        // stencil s = (a, a, a, b, b, b): left from s0..s4, right from s5..s1
        *lp[v] = weno5<Pol>(a, a, a, b, b, eps);
        *rp[v] = weno5<Pol>(b, b, b, a, a, eps);
    }
    finish_state<Pol>(L, g);
    finish_state<Pol>(R, g);
}

// Asynchronous global -> shared copies (cp.async, sm_80+): 16 bytes each,
// bypassing L1, zero filled without reading when `valid` is false (gmem must
// still be a valid address); completion per thread in commit groups.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
// one cell of the stored state (all four variables), zero filled when not valid
template <class T>
__device__ __forceinline__ void cp_async_cell(T* smem, const T* gmem, bool valid) {
    cp_async16(smem, gmem, valid);
    if constexpr (sizeof(T) == 8) cp_async16(smem + 2, gmem + 2, valid);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Ring of staged rows of the row march (load schedules 3 and 4), per warp:
// kRingRows rows of its 36 columns (the segment and 2 halo columns each side,
// whole cells), stored values, and (FP32 storage) the same 36 columns of the
// rows of U^0 (lane l reads column l + 2).  The FP64 ring leaves U^0 out (each
// lane loads it early in the row's iteration): its rows of doubles would
// otherwise cost a fourth block per SM.
// A ring row holds 36 cells and starts 128-byte aligned, as a TMA copy's
// shared-memory destination must: its stride is rounded up to 128 bytes
// (FP32: 576 bytes of cells in a 640-byte row; FP64: 1,152 bytes, already a
// multiple).
constexpr int kRingRows = 8, kRingDist = 2;
constexpr int kRingCols = 36;
template <class T>
__host__ __device__ constexpr int ring_row_words() {
    return ((kRingCols * kVars * static_cast<int>(sizeof(T)) + 127) / 128) * 128 / static_cast<int>(sizeof(T));
}
template <class T>
__host__ __device__ constexpr int ring_words() {
    return sizeof(T) == 4 ? kRingRows * 2 * ring_row_words<T>() : kRingRows * ring_row_words<T>();
}
static_assert(ring_row_words<float>() * 4 % 128 == 0 && ring_row_words<double>() * 8 % 128 == 0,
              "ring rows start 128-byte aligned");
static_assert(ring_words<float>() * 4 % 128 == 0 && ring_words<double>() * 8 % 128 == 0,
              "each warp's ring starts 128-byte aligned");

// ---- TMA staging (load schedule 4).  One elected lane of a warp copies a
// whole ring row -- the 4 variables of 36 cells, one box of the state
// buffer's 3-D tensor map (variables, columns, rows) -- with one bulk tensor
// copy that signals an mbarrier of the row's ring slot; the lanes wait on
// that barrier instead of issuing per-lane copies.  The tensor maps travel in
// the kernel's __grid_constant__ argument block (StageArgs::tmap_in,
// tmap_u0) and cover this GPU's own state buffers only; no copy is
// multicast.  Every wait is bounded: a copy that never lands sets
// *StageArgs::err and ends the work item.
__device__ __forceinline__ unsigned smem_addr(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0u;
}
// try_wait suspends the thread for a system-dependent time per attempt; this
// many attempts is far beyond any copy's latency (a row lands within a few
// microseconds); the drain after a failure tries less
constexpr int kMbarMaxTries = 1 << 20;
constexpr int kMbarDrainTries = 1 << 14;
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity, int tries = kMbarMaxTries) {
    for (int k = 0; k < tries; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// generic-proxy accesses of this thread (and, after a __syncwarp, of its warp)
// before later async-proxy (TMA) writes to shared memory
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tma_load_row(unsigned dst, const void* tmap, int col, int row, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
        ::"r"(dst), "l"(tmap), "r"(0), "r"(col), "r"(row), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma_prefetch_map(const void* tmap) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(tmap) : "memory");
}

// One column's 4 variables to / from the shared row buffer in vector accesses.
template <class C>
__device__ __forceinline__ void put_slot(C (&slot)[kVars], const C v[kVars]) {
    if constexpr (sizeof(C) == 4) {
        *reinterpret_cast<float4*>(slot) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        reinterpret_cast<double2*>(slot)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(slot)[1] = make_double2(v[2], v[3]);
    }
}

template <class C>
__device__ __forceinline__ void get_slot(const C (&slot)[kVars], C v[kVars]) {
    if constexpr (sizeof(C) == 4) {
        const float4 t = *reinterpret_cast<const float4*>(slot);
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    } else {
        const double2 a = reinterpret_cast<const double2*>(slot)[0], b = reinterpret_cast<const double2*>(slot)[1];
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
}

// Positivity fallback of one cell's two reconstructed states in one direction
// (no reference counterpart).  A state is admissible when rho > 0 and p > 0
// (NaN fails); a state that is not, or that lies on a face flagged low order
// (a non-fluid cell in the face's stencil), becomes the cell's own value (first
// order).  `c` is the cell's value; the replacement is finished only when a
// state needs it.
template <class Pol>
__device__ __forceinline__ bool admissible(const Face5<typename Pol::C>& s) {
    return s.r > typename Pol::C(0) && s.p > typename Pol::C(0);
}

template <class Pol>
__device__ __forceinline__ void fix_states(bool lowL, bool lowR, const typename Pol::C c[kVars], double g,
                                           Face5<typename Pol::C>& L, Face5<typename Pol::C>& R) {
    const bool bl = lowL || !admissible<Pol>(L), br = lowR || !admissible<Pol>(R);
    if (bl || br) {
        Face5<typename Pol::C> s;
        s.r = c[0];
        s.mx = c[1];
        s.my = c[2];
        s.E = c[3];
        finish_state<Pol>(s, g);
        if (bl) L = s;
        if (br) R = s;
    }
}

// The same fallback on the two states of a physical boundary face, each taking
// the value of the cell on its side (cl left of the face, cr right of it).
template <class Pol>
__device__ __forceinline__ void fix_face(bool low, const typename Pol::C cl[kVars], const typename Pol::C cr[kVars],
                                         double g, Face5<typename Pol::C>& L, Face5<typename Pol::C>& R) {
    Face5<typename Pol::C> dummy = R;
    fix_states<Pol>(low, false, cl, g, L, dummy);
    dummy = L;
    fix_states<Pol>(false, low, cr, g, dummy, R);
}

// Fluxes through the physical boundary faces of one stage (the reference's
// boundary stencil [g g g | c c c], CellInterface.cpp:172-178, then the
// positivity fallback and HLL), computed by boundary_flux_kernel before the
// row march, which reads them (StageArgs::bflux) instead of reconstructing
// there.
template <class Pol>
__device__ __forceinline__ void boundary_face_flux(const StageArgs& a, int s, int k) {
    using T = typename Pol::T;
    using C = typename Pol::C;
    const Layout& L = a.L;
    const T* in = static_cast<const T*>(a.in);
    // interior cell (ii, jj) and ghost cell (gi, gj) of face k of side s
    int ii, jj, gi, gj;
    if (s < 2) {
        jj = gj = k;
        ii = s == 0 ? 0 : L.nx - 1;
        gi = s == 0 ? -1 : L.nx;
    } else {
        ii = gi = k;
        jj = s == 2 ? 0 : L.ny - 1;
        gj = s == 2 ? -1 : L.ny;
    }
    C c[kVars], gh[kVars];
    T cs[kVars], gs[kVars];
    ld_cell<T>(in, L.offset(ii, jj), cs);
    ld_cell<T>(in, L.offset(gi, gj), gs);
#pragma unroll
    for (int v = 0; v < kVars; ++v) {
        c[v] = decc<T, C>(cs[v], L, v);
        gh[v] = decc<T, C>(gs[v], L, v);
    }
    const bool lo = s == 0 || s == 2;
    Face5<C> Lf, Rf;
    boundary_face_states<Pol>(c, gh, lo, C(a.eps), a.gamma, Lf, Rf);
    if (a.positivity) {
        // face flags [nx+1][ny+1]: bit 0 x-face (i-1/2, j), bit 1 y-face (i, j-1/2)
        bool low = false;
        if (a.lowo) {
            const long long f = s == 0 ? jj : s == 1 ? static_cast<long long>(L.nx) * (L.ny + 1) + jj
                              : s == 2 ? static_cast<long long>(ii) * (L.ny + 1) : static_cast<long long>(ii) * (L.ny + 1) + L.ny;
            low = a.lowo[f] & (s < 2 ? 1 : 2);
        }
        fix_face<Pol>(low, lo ? gh : c, lo ? c : gh, a.gamma, Lf, Rf);
    }
    C F[kVars];
    hll_flux<Pol>(Lf, Rf, s < 2 ? 0 : 1, a.hll, a.gamma, F);
    C* out = static_cast<C*>(a.bflux) + bflux_side_offset(L, s);
    const int n = s < 2 ? L.ny : L.nx;
#pragma unroll
    for (int v = 0; v < kVars; ++v) out[static_cast<long long>(v) * n + k] = F[v];
}

// One thread per boundary face: blockIdx.y = side, threads over the face index.
template <class Pol>
__global__ void __launch_bounds__(128) boundary_flux_kernel(const StageArgs a) {
    const int s = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (!physical_side(a, s) || k >= (s < 2 ? a.L.ny : a.L.nx)) return;
    boundary_face_flux<Pol>(a, s, k);
}

// Batched form: blockIdx.z = case (args[c]), blockIdx.y = side.
template <class Pol>
__global__ void __launch_bounds__(128) batch_boundary_flux_kernel(const StageArgs* __restrict__ args) {
    const StageArgs& a = args[blockIdx.z];
    const int s = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (!a.bflux || !physical_side(a, s) || k >= (s < 2 ? a.L.ny : a.L.nx)) return;
    boundary_face_flux<Pol>(a, s, k);
}

// One work item: rows [by*rows, by*rows + rows) of segment `seg` (columns
// seg*30 .. seg*30+29), one warp.  The warps of a block share nothing but their
// slices of the row buffer and their rings.  kLoad, where global loads
// are issued (the trade is latency hidden against registers held):
//   0 at their use;
//   1 early in the iteration: the next row, the y halo columns and the RK
//     operands right after the row's x reconstruction, ahead of the update and
//     the y work that precede their use;
//   2 ahead: the next row two iterations ahead, the halo columns one row ahead,
//     the RK operands before the x reconstruction;
//   3 staged: every row of the segment (with its halo columns) and, in the
//     FP32 form, of U^0 is copied asynchronously (cp.async) into a per-warp
//     shared ring `ring` kRingDist rows ahead of its use; the x and y stencils,
//     the stored value and (FP32) U^0 of the update are read from the ring, so
//     no row window is held in registers and load latency overlaps rows of
//     arithmetic (the FP64 form loads U^0 early in the row's iteration and
//     keeps its ring in dynamic shared memory).
//
// The row loop holds no rarely taken code of any size: physical boundary faces
// read the fluxes of boundary_flux_kernel and cell types and low-order faces
// come from one flag byte per cell (StageArgs::cflags), both compiled in only
// with kFeatEdge; the positivity fallback is a select of the cell's own state
// (kFeatPos); the RHS copy and viscous RHS come with kFeatExtra.  A loop body that outgrows the
// instruction cache stalls every warp on instruction fetch, whatever the share
// of the rare code actually executed.
template <class Pol, int kWarps, int kLoad, int kFeat>
__device__ __forceinline__ bool march_item(const StageArgs& a, int seg, int by, int rows,
                                           typename Pol::C (&rbuf)[kWarps][36][kVars],
                                           typename Pol::T* ring, int wid, unsigned long long* bars = nullptr,
                                           unsigned* phase = nullptr) {
    using T = typename Pol::T;
    using C = typename Pol::C;
    constexpr bool kTma = kLoad == 4;
    constexpr bool kRing = kLoad >= 3;
    constexpr int kL = kLoad;
    constexpr bool kPos = (kFeat & kFeatPos) != 0;
    constexpr bool kExtra = (kFeat & kFeatExtra) != 0;
    constexpr bool kEdge = (kFeat & kFeatEdge) != 0;
    const Layout& L = a.L;
    const int lane = threadIdx.x & 31;
    const int j0 = seg * kSeg;
    const int i0 = stage_row_lo(a) + by * rows;
    const int i1 = min(i0 + rows, stage_row_hi(a));
    const int j = j0 - 1 + lane;                 // this lane's column
    const bool col_ok = j <= L.ny + kGhost - 1;  // inside the padded row
    const bool owner = lane >= 1 && lane <= kSeg && j < L.ny;  // updates cells of this column
    const T* in = static_cast<const T*>(a.in);
    const C eps = C(a.eps);
    const double g = a.gamma;
    const double dt = stage_dt(a);
    const double inv_dx = 1.0 / a.dx, inv_dy = 1.0 / a.dy;
    const float inv_dxf = float(inv_dx), inv_dyf = float(inv_dy);
    // FP32 update coefficients of this stage: new = cA x0 + cB x1 + (c dt) R with
    // x0 = U^0 (or the current state at stage 0), x1 = U^1 (TVD3 as written,
    // stage 2) or the current state (TVD2rdRK.h:16-19, TVD3rdRK.h:14-18).
    float cA = 1.0f, cB = 0.0f;
    double cdtd = dt;  // dt coefficient of the stage, FP64
    bool x1_u1 = false;
    if (a.stage == 1) {
        if (a.rk == kRkTvd2) { cA = 0.5f; cB = 0.5f; cdtd = 0.5 * dt; }
        else { cA = 0.75f; cB = 0.25f; cdtd = 0.25 * dt; }
    } else if (a.stage == 2) {
        // cA + cB must be exactly 1 in FP32, else the deviation form scales the
        // stored deviations by (cA + cB) every step: cB = fl(2/3), cA = 1 - cB
        // (an exact FP32 subtraction).
        cB = float(2.0 / 3.0);
        cA = 1.0f - cB;
        cdtd = (2.0 / 3.0) * dt;
        x1_u1 = a.rk == kRkTvd3Ref;
    }
    const float cdt = float(cdtd);
    // Stochastic rounding of the state that ends each step (the last stage), or
    // of every stage (CFS_ROUND_STOCHASTIC_ALL); otherwise round to nearest.
    // Rounding an intermediate stage to nearest leaves a small mass bias: its
    // increments are dt times differences of FP32 fluxes, a coarse lattice on
    // the stored grid, so the rounding errors do not average out.
    const bool last_of_step = a.rk == kRkTvd2 ? a.stage == 1 : a.stage == 2;
    const bool sr = Pol::kMixed && ((a.rounding == 0 && last_of_step) || a.rounding == 2);
    const unsigned int step_seed = (a.P ? a.P->seed[a.parity] : a.seed) * 4u + static_cast<unsigned int>(a.stage);
    // physical boundary faces: fluxes precomputed (boundary_flux_kernel)
    const bool lo_x = kEdge && physical_side(a, 0), hi_x = kEdge && physical_side(a, 1);
    const bool lo_y = kEdge && physical_side(a, 2), hi_y = kEdge && physical_side(a, 3);
    const C* const bfl = static_cast<const C*>(a.bflux);
    const uint8_t* const flags = kEdge ? a.cflags : nullptr;
    double* const rhs_out = kExtra ? a.rhs : nullptr;
    const T* const rv_in = kExtra ? static_cast<const T*>(a.rv) : nullptr;
    if (a.P && a.first_stage && seg == 0 && by == 0 && lane == 0) {
        a.P->wmax[1 - a.parity] = 0ull;
        a.P->t += dt;
        a.P->dt_last = dt;
        a.P->seed[1 - a.parity] = a.P->seed[a.parity] + 1u;
    }
    const bool active_warp = j0 < L.ny;  // uniform per warp
    const bool do_cfl = a.P && a.last_stage && a.P->use_cfl;  // read once: stores to `out` may alias P for the compiler

    auto load_row = [&](int r, C out[kVars]) {
        if (col_ok) {
            T cv[kVars];
            ld_cell<T>(in, L.offset(r, j), cv);
#pragma unroll
            for (int v = 0; v < kVars; ++v) out[v] = decc<T, C>(cv[v], L, v);
        } else {
#pragma unroll
            for (int v = 0; v < kVars; ++v) out[v] = C(0);
        }
    };

    auto load_halo = [&](int r, C h[kVars]) {
        if (lane < 2 || lane >= 30) {  // halo columns j0-3, j0-2 and j0+31, j0+32
            const int hc = lane < 2 ? j0 - 3 + lane : j0 + 1 + lane;
            if (hc <= L.ny + kGhost - 1) {
                T cv[kVars];
                ld_cell<T>(in, L.offset(r, hc), cv);
#pragma unroll
                for (int v = 0; v < kVars; ++v) h[v] = decc<T, C>(cv[v], L, v);
            } else {
#pragma unroll
                for (int v = 0; v < kVars; ++v) h[v] = C(0);
            }
        }
    };
    // Flag byte of cell (r, j) (kCell* bits; 0 outside i = -1..nx, j = -1..ny
    // or without flags).
    auto load_flags = [&](int r) -> unsigned int {
        unsigned int f = 0u;
        if (flags && r >= -1 && r <= L.nx) {  // uniform per warp
            if (j <= L.ny) f = flags[static_cast<long long>(r + 1) * (L.ny + 2) + (j + 1)];
        }
        return f;
    };
    // this lane reconstructs the ghost column of a physical y side (its y-face
    // flux is the boundary flux); warp-uniform screen for the rare lanes
    const bool ybnd = (j == -1 && lo_y) || (j == L.ny - 1 && hi_y);
    const bool warp_ybnd = __any_sync(0xffffffffu, ybnd);
    const C* const bfy = ybnd ? bfl + bflux_side_offset(L, j == -1 ? 2 : 3) : nullptr;
    // RK operands of cell (i, j): the stored value (FP32 form), U^0.
    // (U^1, read by the reference's TVD3 stage 2 only, is loaded at its use.)
    T pf_cur[kVars], pf_u0[kVars];
    auto load_update = [&](int i) {
        const long long off = L.offset(i, j);
        if (Pol::kMixed) ld_cell<T>(in, off, pf_cur);
        if (a.stage >= 1) ld_cell<T>(static_cast<const T*>(a.u0), off, pf_u0);
    };

    // Load schedule 3: this warp's ring (rows, and U^0 rows in FP32; ring_words).
    constexpr bool kU0Ring = kRing && sizeof(T) == 4;
    constexpr int kRowWords = ring_row_words<T>();
    T* const rw = kRing ? ring + wid * ring_words<T>() : nullptr;
    T* const ru0 = kU0Ring ? rw + kRingRows * kRowWords : nullptr;
    auto ring_row = [&](int q) -> T* { return rw + (q & (kRingRows - 1)) * kRowWords; };
    auto ring_u0 = [&](int q) -> T* { return ru0 + (q & (kRingRows - 1)) * kRowWords; };
    // Issue the copies of row q (the lane's column; halo lanes also their
    // halo column) and, for an updated row, of its U^0; one commit group per
    // row (empty past the last row needed, so group counts stay uniform).
    // TMA: lane 0 copies the row's 36 cells (and U^0's) as one box each,
    // completing on the slot's mbarrier.
    constexpr unsigned kRowBytes = kRingCols * kVars * sizeof(T);
    const int tcol = L.joff + j0 - 3;  // buffer column of ring column 0 (j0 - 3)
    int issued = i0 - 4;               // TMA: rows <= issued have been issued
    auto issue_row = [&](int q) {
        if constexpr (kTma) {
            if (q > i1 + 2) return;
            issued = q;
            if (lane == 0) {
                const bool u0row = kU0Ring && a.stage >= 1 && q >= i0 && q < i1;
                const unsigned bar = smem_addr(bars + (q & (kRingRows - 1)));
                const unsigned dst = smem_addr(ring_row(q)), dst0 = u0row ? smem_addr(ring_u0(q)) : 0u;
                if (((dst | dst0) & 127u) != 0u) {
                    // self-check: never issue a copy to a misaligned row;
                    // complete the slot's phase without data and flag it
                    atomicOr(a.err, kErrTmaAlign);
                    mbar_arrive(bar);
                } else {
                    fence_proxy_async_smem();
                    mbar_expect_tx(bar, u0row ? 2u * kRowBytes : kRowBytes);
                    tma_load_row(dst, a.tmap_in, tcol, q + kGhost, bar);
                    if (u0row) tma_load_row(dst0, a.tmap_u0, tcol, q + kGhost, bar);
                }
            }
        } else if constexpr (kRing) {
            if (q <= i1 + 2) {
                T* dst = ring_row(q);
                const long long off = L.offset(q, col_ok ? j : 0);
                cp_async_cell<T>(dst + (lane + 2) * kVars, in + Layout::at(off, 0), col_ok);
                if (lane < 2 || lane >= 30) {
                    const int hc = lane < 2 ? j0 - 3 + lane : j0 + 1 + lane;
                    const bool ok = hc <= L.ny + kGhost - 1;
                    const long long hoff = L.offset(q, ok ? hc : 0);
                    const int slot = lane < 2 ? lane : lane + 4;
                    cp_async_cell<T>(dst + slot * kVars, in + Layout::at(hoff, 0), ok);
                }
                if (kU0Ring && a.stage >= 1 && q >= i0 && q < i1)  // uniform: every lane fills its slot
                    cp_async_cell<T>(ring_u0(q) + (lane + 2) * kVars, static_cast<const T*>(a.u0) + Layout::at(off, 0),
                                     col_ok);
            }
            cp_async_commit();
        }
    };
    // TMA: wait until row q has landed in its slot (each row is waited on
    // exactly once, in order, so one phase bit per slot tracks its fills)
    bool tma_ok = true;
    int waited = i0 - 4;  // rows <= waited have been waited on
    auto wait_row = [&](int q) {
        if constexpr (kTma) {
            if (q > i1 + 2 || !tma_ok) return;
            const int sl = q & (kRingRows - 1);
            // warp-uniform outcome: every lane continues or every lane stops
            if (!__all_sync(0xffffffffu, mbar_wait_bounded(smem_addr(bars + sl), (*phase >> sl) & 1u))) {
                tma_ok = false;
                return;
            }
            *phase ^= 1u << sl;
            waited = q;
        }
    };
    // full value of a stencil cell (the ring holds stored deviations)
    auto full = [&](const C w[kVars], C out[kVars]) {
#pragma unroll
        for (int v = 0; v < kVars; ++v) out[v] = (kRing && Pol::kMixed) ? w[v] + C(L.off[v]) : w[v];
    };

    C win[5][kVars];
    C nxt[kVars];   // kLoad 1, 2: the row after win[4]
    C hal[kVars];   // kLoad 1, 2: halo columns of the next y row
    Face5<C> Lx{};                             // left x-state of the previous row
    C FXp[kVars] = {C(0), C(0), C(0), C(0)};   // x-flux through the lower face of the previous row
    C RY[kVars] = {C(0), C(0), C(0), C(0)};    // y part of the previous row's RHS
    unsigned int f_prev = 0u, f_next = 0u;     // flags of rows r-1 and r+1
    T rv_cur[3] = {T(0), T(0), T(0)}, rv_pf[3] = {T(0), T(0), T(0)};  // kExtra: viscous RHS of rows r-1, r
    double wloc = 0.0;
    if (active_warp && kRing) {
        if constexpr (kTma) __syncwarp();  // a previous item's reads of the ring end before lane 0's copies
        for (int q = i0 - 3; q <= i0 + 1 + kRingDist; ++q) issue_row(q);
        if constexpr (kTma) {
            for (int q = i0 - 3; q <= i0; ++q) wait_row(q);  // the first iteration waits for row i0 + 1
        }
    } else if (active_warp) {
#pragma unroll
        for (int k = 0; k < 5; ++k) load_row(i0 - 3 + k, win[k]);
        if constexpr (kL == 2) {
            load_row(i0 + 2, nxt);
            load_halo(i0, hal);
        }
    }
    if (active_warp) f_next = load_flags(i0 - 1);
    for (int r = i0 - 1; active_warp && r <= i1; ++r) {
        const unsigned int f_r = f_next;
        f_next = load_flags(r + 1);
        if constexpr (kRing && !kU0Ring) {  // FP64 ring: U^0 of row r-1, ahead of the x reconstruction
            if (a.stage >= 1 && owner && r - 1 >= i0) ld_cell<T>(static_cast<const T*>(a.u0), L.offset(r - 1, j), pf_u0);
        }
        if constexpr (kExtra) {  // viscous RHS of row r, a whole iteration ahead of its update
#pragma unroll
            for (int q = 0; q < 3; ++q) rv_cur[q] = rv_pf[q];
            if (rv_in && owner && r >= i0 && r < i1) {
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    rv_pf[q] = rv_in[static_cast<long long>(q) * L.nx * L.ny + static_cast<long long>(r) * L.ny + j];
            }
        }
        if constexpr (kRing) {
            // every lane is done with the previous iteration's slots; the slot
            // now refilled held row r+3+kRingDist-kRingRows, last read at r-1
            __syncwarp();
            issue_row(r + 3 + kRingDist);
            if constexpr (kTma) {
                wait_row(r + 2);  // rows <= r+2 have landed
                if (!tma_ok) break;
            } else {
                cp_async_wait<kRingDist + 1>();  // this lane's copies of rows <= r+2 have landed
                __syncwarp();                    // ... and every lane's
            }
#pragma unroll
            for (int k = 0; k < 5; ++k) {  // stored deviations; offsets added after the reconstruction
                const T* src = ring_row(r - 2 + k) + (lane + 2) * kVars;
#pragma unroll
                for (int v = 0; v < kVars; ++v) win[k][v] = C(src[v]);
            }
        }
        if constexpr (kL == 2) {
            if (r - 1 >= i0 && owner) load_update(r - 1);
        }
        // ---- x reconstruction of row r
        Face5<C> Lr, Rr;
        cell_states<Pol>(win, eps, g, Lr, Rr, (kRing && Pol::kMixed) ? L.off : nullptr);
        if constexpr (kPos) {
            C cc[kVars];
            full(win[2], cc);
            fix_states<Pol>(f_r & kCellLowXhi, f_r & kCellLowXlo, cc, g, Lr, Rr);
        }
        if constexpr (kL == 1) {
            if (r < i1) load_row(r + 3, nxt);
            if (r - 1 >= i0 && owner) load_update(r - 1);
            if (r >= i0 && r < i1) load_halo(r, hal);
        }
        C FX[kVars] = {C(0), C(0), C(0), C(0)};
        if (r >= i0) {
            // (computed on a boundary row too and replaced there: a flux in a
            // branch of its own would not overlap the surrounding work)
            hll_flux<Pol>(Lx, Rr, 0, a.hll, g, FX);
            if ((r == 0 && lo_x) || (r == L.nx && hi_x)) {  // uniform per warp
                const C* b = bfl + bflux_side_offset(L, r == 0 ? 0 : 1);
                if (j >= 0 && j < L.ny) {
#pragma unroll
                    for (int v = 0; v < kVars; ++v) FX[v] = b[static_cast<long long>(v) * L.ny + j];
                }
            }
            // ---- update of row r-1 (its upper x-face is r - 1/2)
            const int i = r - 1;
            if (i >= i0 && owner) {
                if constexpr (kRing) {
                    const T* cs = ring_row(i) + (lane + 2) * kVars;
#pragma unroll
                    for (int v = 0; v < kVars; ++v) pf_cur[v] = cs[v];
                    if constexpr (kU0Ring) {
                        // U^0 (stage 0: the current state, the update's x0 then)
                        const T* us = (a.stage >= 1 ? ring_u0(i) : ring_row(i)) + (lane + 2) * kVars;
#pragma unroll
                        for (int v = 0; v < kVars; ++v) pf_u0[v] = us[v];
                    }
                } else if constexpr (kL == 0) {
                    load_update(i);
                }
                const bool fluid = !kEdge || !(f_prev & kCellSolid);
                T* out = static_cast<T*>(a.out);
                T u1c[kVars] = {T(0), T(0), T(0), T(0)};  // U^1 (TVD3 as written, stage 2 only)
                if (a.stage == 2 && a.rk == kRkTvd3Ref) ld_cell<T>(static_cast<const T*>(a.u1), L.offset(i, j), u1c);
                C nv[kVars];  // new state in the form's arithmetic type, for the CFL maximum
                T sv[kVars];
                if constexpr (Pol::kMixed) {
                    // FP32 update of the stored deviations (value - off): the RK
                    // coefficients of a stage sum to 1, so the offsets cancel and
                    // the rounding step is that of the deviation.
                    // (formed for every cell and selected: a non-fluid cell keeps its state)
                    float rvf[kVars], x0[kVars], x1[kVars], ndv[kVars];
#pragma unroll
                    for (int v = 0; v < kVars; ++v) {
                        rvf[v] = -(FX[v] - FXp[v]) * inv_dxf + RY[v];
                        if (kExtra && rv_in && v >= 1) rvf[v] += rv_cur[v - 1];
                        x0[v] = (kU0Ring || a.stage >= 1) ? pf_u0[v] : pf_cur[v];
                        // (stage 0: cB = 0 and x1 - x0 = 0, so x1 adds nothing)
                        x1[v] = x1_u1 ? u1c[v] : pf_cur[v];
                    }
                    if (sr) {
                        // Stochastic rounding of x0 + cB (x1 - x0) + cdt R (cA = 1 - cB
                        // exactly): the increment is formed first, at its own
                        // spacing (roundings near 1e-12 of the state, far below the
                        // stored spacing), gets a dither uniform over one stored
                        // spacing of the result's binade, and is added to x0 with
                        // one rounding; two variables per packed instruction.
                        const unsigned int h = cell_hash(i, j, step_seed);
#pragma unroll
                        for (int v = 0; v < kVars; v += 2) {
                            const float2 a0 = make_float2(x0[v], x0[v + 1]);
                            const float2 inc = fma2(p2(cB), sub2(make_float2(x1[v], x1[v + 1]), a0),
                                                    mul2(p2(cdt), make_float2(rvf[v], rvf[v + 1])));
                            const float2 f = add2(a0, inc);
                            const float2 dz = make_float2(sr_dither(f.x, h >> (8 * v)), sr_dither(f.y, h >> (8 * v + 8)));
                            const float2 r = add2(a0, add2(inc, dz));
                            ndv[v] = r.x;
                            ndv[v + 1] = r.y;
                        }
                    } else {
#pragma unroll
                        for (int v = 0; v < kVars; ++v) ndv[v] = fmaf(cdt, rvf[v], fmaf(cA, x0[v], cB * x1[v]));
                    }
#pragma unroll
                    for (int v = 0; v < kVars; ++v) {
                        const float cur = pf_cur[v];
                        const float nd = fluid ? ndv[v] : cur;
                        sv[v] = nd;
                        nv[v] = nd + L.off[v];
                        if (kExtra && rhs_out)
                            rhs_out[static_cast<long long>(v) * L.nx * L.ny + static_cast<long long>(i) * L.ny + j] = fluid ? double(rvf[v]) : 0.0;
                    }
                } else {
#pragma unroll
                    for (int v = 0; v < kVars; ++v) {
                        double rv = -double(FX[v] - FXp[v]) * inv_dx + double(RY[v]);
                        if (kExtra && rv_in && v >= 1) rv += double(rv_cur[v - 1]);
                        const double cur = double(win[1][v]);
                        const double u0v = a.stage >= 1 ? dec<T>(pf_u0[v], L, v) : 0.0;
                        const double u1v = (a.stage == 2 && a.rk == kRkTvd3Ref) ? dec<T>(u1c[v], L, v) : 0.0;
                        const double val = fluid ? rk_update(a.rk, a.stage, dt, cur, u0v, u1v, rv) : cur;
                        sv[v] = enc<T>(val, L, v);
                        nv[v] = C(dec<T>(sv[v], L, v));
                        if (kExtra && rhs_out)
                            rhs_out[static_cast<long long>(v) * L.nx * L.ny + static_cast<long long>(i) * L.ny + j] = fluid ? rv : 0.0;
                    }
                }
                if (kPos && a.positivity >= kPosFloor && fluid) {
                    // p > floor, multiplied by rho > 0: (g-1)(rho E - |m|^2/2) > floor rho
                    const C q = nv[3] * nv[0] - C(0.5) * (nv[1] * nv[1] + nv[2] * nv[2]);
                    if (!(nv[0] > C(kRhoFloor)) || !(C(g - 1.0) * q > C(kPFloor) * nv[0])) {
                        double s[kVars];
#pragma unroll
                        for (int v = 0; v < kVars; ++v)
                            s[v] = Pol::kMixed ? double(sv[v]) + double(L.off[v]) : double(nv[v]);
                        floor_state(s, g);
#pragma unroll
                        for (int v = 0; v < kVars; ++v) {
                            sv[v] = Pol::kMixed ? T(s[v] - double(L.off[v])) : T(s[v]);
                            nv[v] = C(s[v]);
                        }
                    }
                }
                store_cell4<T>(out, L, a.bc, i, j, sv);
                if (do_cfl) {
                    const double w = cfl_term(double(wave_sum_fast<C>(nv[0], nv[1], nv[2], nv[3], C(g), C(inv_dx), C(inv_dy))));
                    if (fluid && w > wloc) wloc = w;
                }
            }
        }
        // ---- y work of row r
        if (r >= i0 && r < i1) {
            // slot-major row buffer: the 4 variables of a column are one
            // 16-byte (FP32) or two 16-byte (FP64) shared accesses
            C st[5][kVars];
            if constexpr (kRing) {
                const T* row = ring_row(r);
#pragma unroll
                for (int k = 0; k < 5; ++k)
#pragma unroll
                    for (int v = 0; v < kVars; ++v) st[k][v] = C(row[(lane + k) * kVars + v]);  // deviations
            } else {
                C(*rb)[kVars] = rbuf[wid];
                put_slot<C>(rb[lane + 2], win[2]);
                if constexpr (kL == 0) load_halo(r, hal);
                if (lane < 2 || lane >= 30) put_slot<C>(rb[lane < 2 ? lane : lane + 4], hal);
                __syncwarp();
#pragma unroll
                for (int k = 0; k < 5; ++k) get_slot<C>(rb[lane + k], st[k]);
            }
            Face5<C> Ly, Ry;
            cell_states<Pol>(st, eps, g, Ly, Ry, (kRing && Pol::kMixed) ? L.off : nullptr);
            if constexpr (kPos) {
                C cc[kVars];
                full(st[2], cc);
                fix_states<Pol>(f_r & kCellLowYhi, f_r & kCellLowYlo, cc, g, Ly, Ry);
            }
            // right state of the cell above (lane + 1)
            Face5<C> Rn;
            Rn.r = __shfl_down_sync(0xffffffffu, Ry.r, 1);
            Rn.mx = __shfl_down_sync(0xffffffffu, Ry.mx, 1);
            Rn.my = __shfl_down_sync(0xffffffffu, Ry.my, 1);
            Rn.E = __shfl_down_sync(0xffffffffu, Ry.E, 1);
            Rn.p = __shfl_down_sync(0xffffffffu, Ry.p, 1);
            Rn.a = __shfl_down_sync(0xffffffffu, Ry.a, 1);
            Rn.ri = __shfl_down_sync(0xffffffffu, Ry.ri, 1);
            // face between column j and j+1 (face index j+1)
            C FY[kVars];
            hll_flux<Pol>(Ly, Rn, 1, a.hll, g, FY);
            if (warp_ybnd && ybnd) {
#pragma unroll
                for (int v = 0; v < kVars; ++v) FY[v] = bfy[static_cast<long long>(v) * L.nx + r];
            }
#pragma unroll
            for (int v = 0; v < kVars; ++v) {
                const C below = __shfl_up_sync(0xffffffffu, FY[v], 1);
                if constexpr (Pol::kMixed) RY[v] = (below - FY[v]) * inv_dyf;  // as the x part: FP32
                else RY[v] = C(-double(FY[v] - below) * inv_dy);
            }
            __syncwarp();
        }
        // ---- carry to the next row
#pragma unroll
        for (int v = 0; v < kVars; ++v) FXp[v] = FX[v];
        Lx = Lr;
        f_prev = f_r;
        if (!kRing && r < i1) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int v = 0; v < kVars; ++v) win[k][v] = win[k + 1][v];
            if constexpr (kL == 2) {
#pragma unroll
                for (int v = 0; v < kVars; ++v) win[4][v] = nxt[v];
                if (r + 4 <= i1 + 2) load_row(r + 4, nxt);
                if (r + 1 < i1) load_halo(r + 1, hal);
            } else if constexpr (kL == 1) {
#pragma unroll
                for (int v = 0; v < kVars; ++v) win[4][v] = nxt[v];
            } else {
                load_row(r + 3, win[4]);
            }
        }
    }
    if constexpr (kTma) {
        if (!tma_ok) {
            // a copy never landed: report it, and wait (bounded) for the
            // copies still in flight so that none outlives the item
            if (lane == 0) atomicOr(a.err, kErrTmaTimeout);
            for (int q = waited + 1; q <= issued; ++q) {
                const int sl = q & (kRingRows - 1);
                if (__all_sync(0xffffffffu, mbar_wait_bounded(smem_addr(bars + sl), (*phase >> sl) & 1u, kMbarDrainTries)))
                    *phase ^= 1u << sl;
            }
            return false;
        }
    } else if constexpr (kRing) {
        cp_async_wait_all();  // no copy into the ring outlives the item
    }
    // CFL maximum: one atomic per warp (no block barrier, so the warps of a
    // block never wait for each other)
    if (do_cfl) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wloc = fmax(wloc, __shfl_xor_sync(0xffffffffu, wloc, o));
        if (lane == 0 && wloc > 0.0)
            atomicMax(&a.P->wmax[1 - a.parity], static_cast<unsigned long long>(__double_as_longlong(wloc)));
    }
    return true;
}

// Per-warp mbarriers of the TMA ring: initialised once per launch by lane 0,
// made visible to the async proxy before the first copy.
template <int kWarps>
__device__ __forceinline__ void init_ring_bars(unsigned long long (&bars)[kWarps][kRingRows], int wid) {
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < kRingRows; ++k) mbar_init(smem_addr(&bars[wid][k]), 1u);
        mbar_init_fence();
    }
    __syncwarp();
}

template <class Pol, int kRows, int kWarps, int kMinBlocks, int kLoad, int kFeat>
__global__ void __launch_bounds__(32 * kWarps, kMinBlocks) march_kernel(const __grid_constant__ StageArgs a) {
    // rows of this launch's work items: chosen by the launcher (a.rows), or the variant's
    const int rows = a.rows > 0 ? a.rows : kRows;
    // warps numbered over (segment, row chunk), segments fastest, so no block
    // carries idle warps when the segments of a row are not a multiple of its
    // warps; a warp past the last item runs an empty one
    const int nseg = (a.L.ny + kSeg - 1) / kSeg;
    const long long nitems =
        static_cast<long long>(nseg) * ((stage_row_hi(a) - stage_row_lo(a) + rows - 1) / rows);
    const long long gw = static_cast<long long>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
    const int seg = gw < nitems ? static_cast<int>(gw % nseg) : nseg;
    const int by = gw < nitems ? static_cast<int>(gw / nseg) : 0;
    // (the ring forms use no row buffer)
    __shared__ __align__(16) typename Pol::C rbuf[kLoad >= 3 ? 1 : kWarps][36][kVars];
    using RB = typename Pol::C(&)[kWarps][36][kVars];
    const int wid = threadIdx.x >> 5;
    if constexpr (kLoad == 4) {
        __shared__ __align__(8) unsigned long long bars[kWarps][kRingRows];
        init_ring_bars<kWarps>(bars, wid);
        if ((threadIdx.x & 31) == 0) {
            tma_prefetch_map(a.tmap_in);
            if (a.stage >= 1 && sizeof(typename Pol::T) == 4) tma_prefetch_map(a.tmap_u0);
        }
        unsigned phase = 0u;
        if constexpr (sizeof(typename Pol::T) == 4) {
            __shared__ __align__(128) typename Pol::T ring[kWarps * ring_words<typename Pol::T>()];
            march_item<Pol, kWarps, kLoad, kFeat>(a, seg, by, rows, reinterpret_cast<RB>(rbuf), ring, wid,
                                                  bars[wid], &phase);
        } else {
            // FP64 ring: dynamic shared memory, sized at launch
            extern __shared__ __align__(128) unsigned char march_dyn_smem[];
            march_item<Pol, kWarps, kLoad, kFeat>(a, seg, by, rows, reinterpret_cast<RB>(rbuf),
                                                  reinterpret_cast<typename Pol::T*>(march_dyn_smem), wid, bars[wid],
                                                  &phase);
        }
    } else if constexpr (kLoad == 3 && sizeof(typename Pol::T) == 4) {
        __shared__ __align__(128) typename Pol::T ring[kWarps * ring_words<typename Pol::T>()];
        march_item<Pol, kWarps, kLoad, kFeat>(a, seg, by, rows, reinterpret_cast<RB>(rbuf), ring, wid);
    } else if constexpr (kLoad == 3) {
        // FP64 ring: kWarps * ring_words<double>() doubles (36.9 KB for 4
        // warps); dynamic shared memory, sized at launch
        extern __shared__ __align__(128) unsigned char march_dyn_smem[];
        march_item<Pol, kWarps, kLoad, kFeat>(a, seg, by, rows, reinterpret_cast<RB>(rbuf),
                                              reinterpret_cast<typename Pol::T*>(march_dyn_smem), wid);
    } else {
        march_item<Pol, kWarps, kLoad, kFeat>(a, seg, by, rows, rbuf, nullptr, threadIdx.x >> 5);
    }
}

// Persistent batched form: one launch runs one stage of every case of a batch.
// Each warp pulls work units (case, segment, row chunk) from a global counter,
// largest cases first, until none are left; warps share nothing, so a case
// whose segment count is not a multiple of the block's warps leaves no warp
// idle.  args[c] holds case c's stage arguments (its own layout, boundaries,
// buffers, dt slot); rows[c] is its row chunk, nseg[c] its segment count.
template <class Pol, int kWarps, int kMinBlocks, int kLoad, int kFeat>
__global__ void __launch_bounds__(32 * kWarps, kMinBlocks)
    batch_march_kernel(const StageArgs* __restrict__ args, const int* __restrict__ unit_case,
                       const int* __restrict__ unit_local, const int* __restrict__ case_rows,
                       const int* __restrict__ case_nseg, int total, unsigned int* counter) {
    using C = typename Pol::C;
    __shared__ __align__(16) C rbuf[kWarps][36][kVars];
    constexpr bool kRing = kLoad == 3;
    constexpr bool kDynRing = kRing && sizeof(typename Pol::T) == 8;  // FP64: ring in dynamic shared memory
    __shared__ __align__(128) typename Pol::T ring_static[kRing && !kDynRing ? kWarps * ring_words<typename Pol::T>() : 1];
    extern __shared__ __align__(128) unsigned char batch_dyn_smem[];
    typename Pol::T* const ring = kDynRing ? reinterpret_cast<typename Pol::T*>(batch_dyn_smem) : ring_static;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    C(&wbuf)[1][36][kVars] = *reinterpret_cast<C(*)[1][36][kVars]>(&rbuf[wid]);
    for (;;) {
        unsigned int w = 0u;
        if (lane == 0) w = atomicAdd(counter, 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w >= static_cast<unsigned int>(total)) break;
        const int c = unit_case[w], lu = unit_local[w];
        const int ns = case_nseg[c];
        const StageArgs a = args[c];
        march_item<Pol, 1, kLoad, kFeat>(a, lu % ns, lu / ns, case_rows[c], wbuf, kRing ? ring + wid * ring_words<typename Pol::T>() : nullptr, 0);
    }
}

}  // namespace cfs
