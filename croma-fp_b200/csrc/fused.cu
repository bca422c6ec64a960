// fused.cu -- the fused FP64 evolve: one warp per (tracer, species)
// system, the spectrum held in registers across a coefficient segment.
//
// Per segment slot and system the warp
//   1. evaluates the loss / diffusion terms of every bin and the Chang-Cooper
//      face weights in rolled, lane-strided loops into the warp's slice of
//      shared memory (losses / Dpp / CC assembly of
//      src/fp_shared_core.c:729-842, 1241-1317, 2358-2431 and
//      src/Chang_Cooper.c:22-184);
//   2. assembles its rows a, b, c in registers -- lane l owns rows
//      [l*R, (l+1)*R), R = nb/32 -- and factors the tridiagonal matrix once,
//      since it is constant over the segment's sub-steps: the Thomas pivots
//      d_i = b_i - a_i c_{i-1}/d_{i-1} are a chain of Moebius maps, composed
//      per lane as 2x2 matrices and combined across lanes by a warp scan; each
//      lane then re-runs the exact recurrence on its rows from the scanned
//      incoming pivot;
//   3. runs every sub-step as the two first-order linear recurrences of
//      fp_thomas_solve_ws (src/fp_shared_core.c:226-257), each an affine warp
//      scan: a local pass per lane, five shuffle levels, a second local pass.
//
// Shared-memory rows are stored at (m % R) * 33 + m / R, so the blocked reads
// of step 2 (lane l, row l*R + r and its neighbours) hit 32 distinct banks.
// Divisions by grid quantities use reciprocals tabulated on the host; the
// results agree with the reference's divisions to an ulp per operation.
// The secondary-electron source of each segment (a dense [tracers x nb] .
// [nb x nb] product, prepare_secondary_sources_cell_major,
// src/fp_shared_core.c:1591-1672) runs as a tiled kernel before the slot.
// Spectra are cell-major [tracer][nb] so that a warp's rows are contiguous.
#include "croma_segment.cuh"

namespace croma {

namespace {

constexpr int kR = NB / 32;          // rows per lane
constexpr int kSw = 33 * kR;         // swizzled row-array length
constexpr int kWarps = 4;            // warps (systems) per block
constexpr unsigned kFull = 0xffffffffu;

struct FusedParams {
    SnapArgs a;              // spectra and sources cell-major [tracer][nb]
    GridTables gt;
    ModelParams mp;
    int slot;
    const double *inje;      // [tracer][nb] electron source of the slot, or null
    const double *eta_scale; // [tracer] Dpp eta-cap scale of the slot, or null (no cap)
    const int *np_min_qe;    // [nb]
    // One caller-defined segment shared by every tracer (run_tracer_pipeline):
    // when set, ex replaces the per-tracer schedule.
    int explicit_seg;
    SegInfo ex;
    // IC rows: shared row (stride 0) or per tracer, momentum-major
    // [nb][ntracer] (stride = ntracer)
    int ic_stride;
};

__device__ __forceinline__ SegInfo segment_of(const FusedParams &P, int t)
{
    return P.explicit_seg ? P.ex : seg_info(P.a.sched, t, P.slot, P.a.dt_snap);
}

__device__ __forceinline__ int swz(int m) { return (m % kR) * 33 + m / kR; }
__device__ __forceinline__ double sup(double v, int d) { return __shfl_up_sync(kFull, v, d); }
__device__ __forceinline__ double sdn(double v, int d) { return __shfl_down_sync(kFull, v, d); }

// Exact power-of-two rescaling of a 2x2 matrix (projective maps are
// unchanged by a common factor).
__device__ __forceinline__ void rescale2(double &m00, double &m01, double &m10, double &m11)
{
    const double mx = fmax(fmax(fabs(m00), fabs(m01)), fmax(fabs(m10), fabs(m11)));
    const long long ex = (__double_as_longlong(mx) >> 52) & 0x7ff;
    if (ex <= 0 || ex >= 2046) return;
    const double sc = __longlong_as_double((2046LL - ex) << 52);
    m00 *= sc; m01 *= sc; m10 *= sc; m11 *= sc;
}

// Per-tracer constants of species S for one segment.
template <int S>
struct SegTerms {
    const GridTables *gt;
    double n_gas, kbt, inv_kbt, inv_n, adiab;
    double synch_coeff, coulomb_coeff;
    double dt, dt_over_tloss_pref;   // protons: dt / T = sig_eff * dt_over_tloss_pref
    double dtT_e;                    // electrons: dt / 1e100
    double dpp_inv, dpp_scale;
    int dpp_fill;
    const double *ric, *ric_next;   // already offset to this tracer
    int ric_stride;                 // bin stride of the IC row
    double alpha;
    int interp;

    // B = radp - 2 Dpp / p, C = Dpp, dT = dt / tloss at bin j
    __device__ __forceinline__ void at(int j, double &B, double &C, double &dT) const
    {
        const SpeciesTables &st = gt->s[S];
        const double p = st.p[j];
        const double p2 = st.p2[j];
        double D;
        if (!dpp_fill) D = p2 * (1.0 / (4.0 * 1.0e+5));
        else if (S == 0) D = p2 * dpp_inv * st.expE[j] * st.exp_cut[j];
        else D = p2 * dpp_inv * st.exp_cut[j];
        D *= dpp_scale;
        double radp;
        if (S == 0) {
            const double xp = gt->cp_Ep[j] * inv_kbt;
            const double xe = xp * (kMe / kMp);
            const double sum = coulomb_kernel_fast(xe) + coulomb_kernel_fast(xp) * (kMe / kMp);
            const double thermal = 1.0 - kbt * gt->cp_inv2mpkin[j];
            const double coul = (thermal < 0.0)
                ? 0.0
                : kGyr * kC / (kMp * kGeV) * sum * n_gas * gt->cp_inv_betap2[j] * thermal * 3.5e-29;
            radp = coul + adiab * p;
            dT = gt->sig_eff[j] * dt_over_tloss_pref;
        } else {
            const double r0 = ric[j * ric_stride];
            const double r = interp ? lerp(r0, ric_next[j * ric_stride], alpha) : r0;
            const double coulomb = coulomb_coeff * (1.0 + log(p * inv_n) * (1.0 / 74.8)) * gt->ce_inv_beta2[j];
            radp = synch_coeff * p2 + r + coulomb + adiab * p;
            dT = dtT_e;
        }
        B = radp - st.two_over_p[j] * D;
        C = D;
    }
};

template <int S>
__device__ __forceinline__ SegTerms<S> seg_terms(const GridTables &gt, const Bg &bg, int dis,
                                                 const SnapArgs &a, const SegInfo &g, int t,
                                                 int ic_stride)
{
    SegTerms<S> T;
    T.gt = &gt;
    T.n_gas = bg.n_gas;
    T.kbt = bg.kbt;
    T.inv_kbt = 1.0 / bg.kbt;
    T.inv_n = 1.0 / bg.n_gas;
    T.adiab = 1.0 / 3.0 * (dis ? 0.0 : bg.divv);
    const double b_ratio = bg.b_field * 1.0e+6 / 3.2;
    T.synch_coeff = 4.8e-4 * b_ratio * b_ratio * 9.11e-28 * 3.0e+10 * 3.1536e+16;
    T.coulomb_coeff = 3.05e-29 * bg.n_gas * kC * kGyr / (kMe * kGeV);
    T.dt = g.dt;
    T.dt_over_tloss_pref = g.dt / (1.0 / (0.5 * kC * bg.n_gas) / kGyr);
    T.dtT_e = g.dt / 1.0e+100;
    T.ric = a.ic_curr + (ic_stride ? t : 0);
    T.ric_next = a.ic_next + (ic_stride ? t : 0);
    T.ric_stride = ic_stride ? ic_stride : 1;
    T.alpha = g.alpha;
    T.interp = g.nseg > 1;
    T.dpp_inv = 0.0;
    T.dpp_scale = 1.0;
    T.dpp_fill = 0;
    return T;
}

struct WarpSmem {
    double B[kSw], C[kSw], D[kSw], Wp[kSw], Wm[kSw];
};

// The factored matrix of one system, distributed over the warp.
template <bool SRC>
struct Factor {
    double inv[kR];      // 1 / d_i
    double h[kR];        // a_i / d_i      (forward recurrence)
    double q[kR];        // c_i / d_i      (back substitution)
    double sd[SRC ? kR : 1];  // dt * source_i / d_i
    double hk[5], qk[5]; // warp-scan multipliers per level
};

// Terms, faces, rows and the factorisation of one system.
template <int S, bool SRC>
__device__ unsigned factorize(const SegTerms<S> &T, const double *sdt, int lane, WarpSmem &sm,
                              Factor<SRC> &F)
{
    const SpeciesTables &st = T.gt->s[S];
    const double *x = st.p;
    unsigned err = 0;

    // terms, lane-strided
#pragma unroll 1
    for (int k = 0; k < kR; k++) {
        const int j = k * 32 + lane;
        double B, C, D;
        T.at(j, B, C, D);
        sm.B[swz(j)] = B;
        sm.C[swz(j)] = C;
        sm.D[swz(j)] = D;
    }
    __syncwarp();
    // faces j (between bins j and j+1), lane-strided
#pragma unroll 1
    for (int k = 0; k < kR; k++) {
        const int j = k * 32 + lane;
        double wp = 0.0, wm = 0.0;
        if (j <= NB - 2) {
            const double cl = sm.C[swz(j)];
            if (fabs(cl) > 1.0e-200) {
                const double w = (sm.B[swz(j)] + sm.B[swz(j + 1)]) / (cl + sm.C[swz(j + 1)]) *
                                 (x[j + 1] - x[j]);
                face_weights(w, wp, wm);
            }
        }
        sm.Wp[swz(j)] = wp;
        sm.Wm[swz(j)] = wm;
    }
    __syncwarp();

    // rows a, b, c of this lane (cc_build_{left,interior,right}, Chang_Cooper.c:66-184)
    const int row0 = lane * kR;
    double A[kR], Bd[kR], Cc[kR];
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const int m = row0 + r;
        const double k = T.dt * st.inv_dx[m];
        const double Cm = sm.C[r * 33 + lane], Bm = sm.B[r * 33 + lane], Dm = sm.D[r * 33 + lane];
        double av = 0.0, bv, cv = 0.0;
        if (m == 0) {
            const double nC = sm.C[swz(1)], nB = sm.B[swz(1)];
            if (fabs(Cm) > 1.0e-200) {
                const double cm12 = 0.5 * (Cm + nC) * st.inv_dxr[0];
                bv = 1.0 + k * (0.0 + cm12 * sm.Wm[swz(0)]) + Dm;
                cv = k * cm12 * sm.Wp[swz(0)];
            } else {
                bv = 1.0 + k * 0.0 + Dm;
                cv = k * 1.0 * 0.5 * (Bm + nB);
            }
        } else {
            const double pC = sm.C[swz(m - 1)], pB = sm.B[swz(m - 1)];
            const double wpm = sm.Wp[swz(m - 1)], wmm = sm.Wm[swz(m - 1)];
            if (m == NB - 1) {
                if (fabs(Cm) > 1.0e-200) {
                    const double cm_12 = 0.5 * (Cm + pC) * st.inv_dxl[m];
                    av = k * cm_12 * wmm;
                    bv = 1.0 + k * (cm_12 * wpm) + Dm;
                    if (isnan(av)) err |= kErrCcNan;
                } else {
                    double dlt = 0.0;
                    if (fabs(pC) > 1.0e-200)
                        dlt = face_delta((pB + Bm) / (pC + Cm) * (x[m] - x[m - 1]));
                    av = -dlt * 0.5 * (Bm + pB) * k;
                    bv = 1.0 + k * (0.5 * (pB + Bm)) + Dm;
                }
            } else {
                const double nC = sm.C[swz(m + 1)], nB = sm.B[swz(m + 1)];
                if (fabs(Cm) > 1.0e-200) {
                    const double cm_12 = 0.5 * (Cm + pC) * st.inv_dxl[m];
                    const double cm12 = 0.5 * (Cm + nC) * st.inv_dxr[m];
                    av = k * cm_12 * wmm;
                    bv = 1.0 + k * (cm_12 * wpm + cm12 * sm.Wm[swz(m)]) + Dm;
                    cv = k * cm12 * sm.Wp[swz(m)];
                } else {
                    // interior row below the diffusion floor: every delta the
                    // reference reads here is zero (Chang_Cooper.c:91-103)
                    bv = 1.0 + k * (0.5 * (Bm + pB)) + Dm;
                    cv = k * 1.0 * 0.5 * (Bm + nB);
                }
            }
        }
        A[r] = av;
        Bd[r] = bv;
        Cc[r] = cv;
    }
    __syncwarp();

    // ---- pivots: composed Moebius maps d -> b - a c_prev / d ----
    const double c_in = sup(Cc[kR - 1], 1);   // c of the row before this lane's first
    double t00 = 1.0, t01 = 0.0, t10 = 0.0, t11 = 1.0;
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const double cprev = (r > 0) ? Cc[r - 1] : (lane > 0 ? c_in : 0.0);
        const double e = A[r] * cprev;
        const double n00 = Bd[r] * t00 - e * t10;
        const double n01 = Bd[r] * t01 - e * t11;
        t10 = t00;
        t11 = t01;
        t00 = n00;
        t01 = n01;
        if ((r & 3) == 3) rescale2(t00, t01, t10, t11);
    }
    rescale2(t00, t01, t10, t11);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) {
        const int off = 1 << lv;
        const double u00 = sup(t00, off), u01 = sup(t01, off), u10 = sup(t10, off), u11 = sup(t11, off);
        if (lane >= off) {
            const double n00 = t00 * u00 + t01 * u10, n01 = t00 * u01 + t01 * u11;
            const double n10 = t10 * u00 + t11 * u10, n11 = t10 * u01 + t11 * u11;
            t00 = n00; t01 = n01; t10 = n10; t11 = n11;
            rescale2(t00, t01, t10, t11);
        }
    }
    double vp = sup(t00, 1), vq = sup(t10, 1);
    double cp_prev = (lane == 0) ? 0.0 : -c_in * vq / vp;
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const int m = row0 + r;
        const double den = Bd[r] + A[r] * cp_prev;
        if (fabs(den) <= 1.0e-300) err |= kErrSingular;
        const double inv = 1.0 / den;
        F.inv[r] = inv;
        F.h[r] = A[r] * inv;
        F.q[r] = (m == NB - 1) ? 0.0 : Cc[r] * inv;
        if (SRC) F.sd[r] = sdt[r] * inv;
        cp_prev = -Cc[r] * inv;
    }

    // ---- warp-scan multipliers of the two linear recurrences ----
    double H = 1.0, Q = 1.0;
#pragma unroll
    for (int r = 0; r < kR; r++) {
        H *= F.h[r];
        Q *= F.q[r];
    }
#pragma unroll
    for (int lv = 0; lv < 5; lv++) {
        const int off = 1 << lv;
        F.hk[lv] = H;
        F.qk[lv] = Q;
        const double Hu = sup(H, off), Qd = sdn(Q, off);
        if (lane >= off) H *= Hu;
        if (lane + off < 32) Q *= Qd;
    }
    (void)vp;
    return err;
}

// One implicit sub-step: N <- M^{-1} (N + dt src) with the factored M.
template <bool SRC>
__device__ __forceinline__ void substep(const Factor<SRC> &F, int lane, double N[kR])
{
    double y[kR];
    double acc = 0.0;
#pragma unroll
    for (int r = 0; r < kR; r++) {
        y[r] = SRC ? fma(N[r], F.inv[r], F.sd[r]) : N[r] * F.inv[r];
        acc = fma(F.h[r], acc, y[r]);
    }
#pragma unroll
    for (int lv = 0; lv < 5; lv++) {
        const int off = 1 << lv;
        const double o = sup(acc, off);
        if (lane >= off) acc = fma(F.hk[lv], o, acc);
    }
    double prev = sup(acc, 1);
    if (lane == 0) prev = 0.0;
#pragma unroll
    for (int r = 0; r < kR; r++) {
        prev = fma(F.h[r], prev, y[r]);
        y[r] = prev;
    }
    acc = 0.0;
#pragma unroll
    for (int r = kR - 1; r >= 0; r--) acc = fma(F.q[r], acc, y[r]);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) {
        const int off = 1 << lv;
        const double o = sdn(acc, off);
        if (lane + off < 32) acc = fma(F.qk[lv], o, acc);
    }
    prev = sdn(acc, 1);
    if (lane == 31) prev = 0.0;
#pragma unroll
    for (int r = kR - 1; r >= 0; r--) {
        prev = fma(F.q[r], prev, y[r]);
        N[r] = prev;
    }
}

// Systems of species S for tracers with a segment in this slot: warp w of
// block b handles tracer b * kWarps + w.
template <int S, bool SRC>
__global__ void __launch_bounds__(kWarps * 32, (NB <= 256 ? 4 : 2)) fused_slot_kernel(FusedParams P)
{
    extern __shared__ double4 smem_raw[];
    WarpSmem *smem = reinterpret_cast<WarpSmem *>(smem_raw);
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const SnapArgs &a = P.a;
    const int t = blockIdx.x * kWarps + w;
    if (t >= a.ntracer) return;
    const SegInfo g = segment_of(P, t);
    if (!g.active) return;
    const Bg bg = load_bg(a, t, g);
    const double tacc = segment_tacc(P.mp, a, g);
    const int dis = a.dis ? a.dis[t] : 0;
    SegTerms<S> T = seg_terms<S>(P.gt, bg, dis, a, g, t, P.ic_stride);
    const int row0 = lane * kR;

    double *Nrow = (S == 0 ? a.crp : a.cre) + (size_t)t * NB + row0;
    double N[kR];
#pragma unroll
    for (int r = 0; r < kR; r += 2) {
        const double2 v = *reinterpret_cast<const double2 *>(Nrow + r);
        N[r] = v.x;
        N[r + 1] = v.y;
    }
    double sdt[SRC ? kR : 1];
    if (SRC) {
        const double *src = (S == 0) ? a.qpi : (P.inje ? P.inje : a.qepri);
#pragma unroll
        for (int r = 0; r < kR; r++) sdt[r] = g.dt * src[(size_t)t * NB + row0 + r];
    }

    const DppForm on = dpp_form(P.mp, P.mp.dpp_model, bg, tacc);
    const double on_scale = (P.mp.dpp_model != kDppOff && P.eta_scale) ? P.eta_scale[t] : 1.0;

    Factor<SRC> F;
    int cur = -1;
    unsigned err = 0;
#pragma unroll 1
    for (int istep = 0; istep < g.steps; istep++) {
        const int want = (!g.windowed || (istep >= g.sl && istep < g.el)) ? 0 : 1;
        if (want != cur) {
            T.dpp_fill = want == 0 ? on.fill : 0;
            T.dpp_inv = want == 0 ? on.inv : 0.0;
            T.dpp_scale = want == 0 ? on_scale : 1.0;
            err |= factorize<S, SRC>(T, sdt, lane, smem[w], F);
            cur = want;
        }
        substep<SRC>(F, lane, N);
    }
    if (err && lane == 0) atomicOr(a.err, err);
#pragma unroll
    for (int r = 0; r < kR; r += 2)
        *reinterpret_cast<double2 *>(Nrow + r) = make_double2(N[r], N[r + 1]);
}

// Dpp eta-cap scale of every tracer with a segment in this slot, from the
// spectra at the start of the segment (prepare_momentumdiff_cell_major,
// src/fp_shared_core.c:1032-1081, runs before either species evolves), one
// warp per tracer.  The energy sum is split over the lanes and combined by a
// shuffle tree, so it agrees with the reference's sequential sum to rounding.
__global__ void __launch_bounds__(128) eta_scale_kernel(FusedParams P, double *eta)
{
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * 4 + (threadIdx.x >> 5);
    const SnapArgs &a = P.a;
    if (t >= a.ntracer) return;
    const SegInfo g = segment_of(P, t);
    if (!g.active) return;
    const Bg bg = load_bg(a, t, g);
    const double tacc_direct = segment_tacc(P.mp, a, g);
    const double mass = a.mass ? a.mass[t] : 0.0;
    const double *crp = a.crp + (size_t)t * NB, *cre = a.cre + (size_t)t * NB;
    double ecr = 0.0;
    for (int j = 2 + lane; j < NB - 2; j += 32) {
        const double ekp = P.gt.s[0].E[j] - kMp, vp = crp[j];
        if (ekp > 0.0 && isfinite(vp)) ecr += ekp * kGeV * vp * P.gt.s[0].dp[j];
        const double eke = P.gt.s[1].E[j] - kMe, ve = cre[j];
        if (eke > 0.0 && isfinite(ve)) ecr += eke * kGeV * ve * P.gt.s[1].dp[j];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ecr += __shfl_xor_sync(kFull, ecr, off);
    if (lane == 0) eta[t] = eta_cap_scale_from_ecr(P.mp, bg, mass, tacc_direct, ecr);
}

// Secondary source of the slot, cell-major:
// inje[t][je] = Gyr n_gas(t) sum_{jp} N_p[t][jp] fqe[jp][je] + qepri[t][je].
// 64 x 64 output tile, 16 x 16 threads, 4 x 4 outputs each; the proton
// index runs upward from the first bin with a nonzero weight in the tile.
__global__ void __launch_bounds__(256) fused_secondary_kernel(FusedParams P, double *inje)
{
    __shared__ double sN[64][17];
    __shared__ double sF[16][64];
    const SnapArgs &a = P.a;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 16 + tx;
    const int t0 = blockIdx.x * 64, je0 = blockIdx.y * 64;
    int jstart = NB;
    for (int i = 0; i < 64 && je0 + i < NB; i++) jstart = min(jstart, P.np_min_qe[je0 + i]);
    jstart = max(jstart, P.gt.fqe_jp0);
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
    for (int k0 = jstart; k0 < NB; k0 += 16) {
        for (int q = tid; q < 64 * 16; q += 256) {
            const int tt = q / 16, kk = q % 16;
            const int t = t0 + tt, jp = k0 + kk;
            sN[tt][kk] = (t < a.ntracer && jp < NB) ? a.crp[(size_t)t * NB + jp] : 0.0;
            const int r = q / 64, col = q % 64;
            const int jp2 = k0 + r;
            sF[r][col] = (jp2 < NB && je0 + col < NB) ? P.gt.fqe[(size_t)jp2 * NB + je0 + col] : 0.0;
        }
        __syncthreads();
        const int kmax = min(16, NB - k0);
        for (int kk = 0; kk < kmax; kk++) {
            double n[4], f[4];
#pragma unroll
            for (int i = 0; i < 4; i++) n[i] = sN[ty + 16 * i][kk];
#pragma unroll
            for (int j = 0; j < 4; j++) f[j] = sF[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fma(n[i], f[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int t = t0 + ty + 16 * i;
        if (t >= a.ntracer) continue;
        const SegInfo g = segment_of(P, t);
        if (!g.active) continue;
        const double ng = (g.nseg > 1) ? lerp(a.bg_curr[t], a.bg_next[t], g.alpha) : a.bg_curr[t];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int je = je0 + tx + 16 * j;
            if (je >= NB) continue;
            const double q = a.qepri ? a.qepri[(size_t)t * NB + je] : 0.0;
            inje[(size_t)t * NB + je] = acc[i][j] * kGyr * ng + q;
        }
    }
}

template <int S, bool SRC>
cudaError_t launch_one(Context &ctx, const FusedParams &P)
{
    constexpr size_t smem = kWarps * sizeof(WarpSmem);
    static bool configured = false;   // per instantiation; set before the first launch
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(fused_slot_kernel<S, SRC>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const int blocks = (P.a.ntracer + kWarps - 1) / kWarps;
    fused_slot_kernel<S, SRC><<<blocks, kWarps * 32, smem, ctx.stream>>>(P);
    return cudaGetLastError();
}

template <int S>
cudaError_t launch_slot(Context &ctx, const FusedParams &P, bool src)
{
    return src ? launch_one<S, true>(ctx, P) : launch_one<S, false>(ctx, P);
}

}  // namespace

int fused_reserve(Context &ctx, int cap)
{
    cudaFree(ctx.d_inje);
    cudaFree(ctx.d_eta_scale);
    ctx.d_inje = ctx.d_eta_scale = nullptr;
    CROMA_CUDA(cudaMalloc(&ctx.d_inje, (size_t)NB * cap * sizeof(double)));
    CROMA_CUDA(cudaMalloc(&ctx.d_eta_scale, (size_t)cap * sizeof(double)));
    return 0;
}

// One slot: the secondary source (when both species evolve), then the
// proton and electron systems.
static int fused_one_slot(Context &ctx, FusedParams &P)
{
    const SnapArgs &a = P.a;
    const int protons = ctx.mp.species_mask & CROMA_SPECIES_PROTON;
    const int electrons = ctx.mp.species_mask & CROMA_SPECIES_ELECTRON;
    cudaEvent_t ev = nullptr;
    P.inje = nullptr;
    P.eta_scale = nullptr;
    if (ctx.mp.eta_dpp_cap > 0.0 && isfinite(ctx.mp.eta_dpp_cap) && ctx.mp.dpp_model != kDppOff) {
        timed_begin(ctx, kKindCoeff, &ev);
        eta_scale_kernel<<<(a.ntracer + 3) / 4, 128, 0, ctx.stream>>>(P, ctx.d_eta_scale);
        timed_end(ctx, kKindCoeff, ev);
        ctx.last_launches += 1;
        P.eta_scale = ctx.d_eta_scale;
    }
    if (protons && electrons) {
        dim3 sg((a.ntracer + 63) / 64, (NB + 63) / 64), sb(16, 16);
        timed_begin(ctx, kKindSecondary, &ev);
        fused_secondary_kernel<<<sg, sb, 0, ctx.stream>>>(P, ctx.d_inje);
        timed_end(ctx, kKindSecondary, ev);
        ctx.last_launches += 1;
        P.inje = ctx.d_inje;
    }
    timed_begin(ctx, kKindEvolve, &ev);
    if (protons) {
        CROMA_CUDA(launch_slot<0>(ctx, P, a.qpi != nullptr));
        ctx.last_launches += 1;
    }
    if (electrons) {
        CROMA_CUDA(launch_slot<1>(ctx, P, P.inje != nullptr || a.qepri != nullptr));
        ctx.last_launches += 1;
    }
    timed_end(ctx, kKindEvolve, ev);
    CROMA_CUDA(cudaGetLastError());
    return 0;
}

int run_fused(Context &ctx, const SnapArgs &a)
{
    FusedParams P;
    P.a = a;
    P.gt = ctx.gt;
    P.mp = ctx.mp;
    P.np_min_qe = ctx.d_np_min_qe;
    P.explicit_seg = 0;
    P.ex = SegInfo{};
    P.ic_stride = 0;
    const int nslots = ctx.mp.interp_max_segments < 1 ? 1 : ctx.mp.interp_max_segments;
    for (int slot = 0; slot < nslots && slot < 64; slot++) {
        P.slot = slot;
        int rc = fused_one_slot(ctx, P);
        if (rc) return rc;
    }
    return 0;
}

int run_fused_segment(Context &ctx, const SnapArgs &a, const SegInfo &ex, int ic_stride)
{
    FusedParams P;
    P.a = a;
    P.gt = ctx.gt;
    P.mp = ctx.mp;
    P.np_min_qe = ctx.d_np_min_qe;
    P.slot = 0;
    P.explicit_seg = 1;
    P.ex = ex;
    P.ic_stride = ic_stride;
    return fused_one_slot(ctx, P);
}

}  // namespace croma
