// fused.cu -- the fused FP64 evolve: one warp per (tracer, species)
// system, the spectrum held in registers across a coefficient segment.
//
// Per segment slot and system the warp
//   1. builds its Chang-Cooper rows on chip: lane l owns rows
//      [l*R, (l+1)*R) (R = nb/32); neighbouring terms and face weights come
//      from the adjacent lanes by shuffles (losses / Dpp / CC assembly of
//      src/fp_shared_core.c:729-842, 1241-1317, 2358-2431 and
//      src/Chang_Cooper.c:22-184);
//   2. factors the tridiagonal matrix once (it is constant over the
//      segment's sub-steps): the Thomas pivots d_i = b_i - a_i c_{i-1}/d_{i-1}
//      are a chain of Moebius maps, composed per lane as 2x2 matrices and
//      combined across lanes by a warp scan; each lane then re-runs the
//      exact recurrence on its rows from the scanned incoming pivot;
//   3. runs every sub-step as two first-order linear recurrences (forward
//      elimination and back substitution of fp_thomas_solve_ws,
//      src/fp_shared_core.c:226-257), each an affine warp scan: a local pass
//      per lane, five shuffle levels, and a second local pass.
//
// The secondary-electron source of each segment (a dense [tracers x nb] .
// [nb x nb] product, prepare_secondary_sources_cell_major,
// src/fp_shared_core.c:1591-1672) runs as a tiled kernel before the slot.
// Spectra are cell-major [tracer][nb] so that a warp's rows are contiguous.
#include "croma_segment.cuh"

namespace croma {

namespace {

constexpr int kRpl = NB / 32;   // rows per lane
constexpr unsigned kFull = 0xffffffffu;

struct FusedParams {
    SnapArgs a;              // spectra and sources cell-major [tracer][nb]
    GridTables gt;
    ModelParams mp;
    int slot;
    const double *inje;      // [tracer][nb] electron source of the slot, or null
    const int *np_min_qe;    // [nb]
};

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

// The factored matrix of one system, distributed over the warp.
struct Factor {
    double inv[kRpl];    // 1 / d_i
    double h[kRpl];      // a_i / d_i      (forward recurrence)
    double q[kRpl];      // c_i / d_i      (back substitution)
    double sd[kRpl];     // dt * source_i / d_i
    double hk[5], qk[5]; // warp-scan multipliers per level
};

// Rows of the lane, then the factorisation.  Returns nonzero error bits.
__device__ unsigned factorize(const SpeciesTerms &T, const double *src_dt, int lane, Factor &F)
{
    const SpeciesTables &st = T.gt->s[T.s];
    const double *x = st.p, *dx = st.dp;
    const double dt = T.dt;
    const int row0 = lane * kRpl;
    unsigned err = 0;

    double B[kRpl], C[kRpl], dT[kRpl];
#pragma unroll
    for (int r = 0; r < kRpl; r++) {
        const Terms tt = T.at(row0 + r);
        B[r] = tt.B;
        C[r] = tt.C;
        dT[r] = tt.dtT;
    }
    const double Bn = sdn(B[0], 1), Cn = sdn(C[0], 1);
    const double Bp = sup(B[kRpl - 1], 1), Cp = sup(C[kRpl - 1], 1);

    // faces j = row0 + r, between bins j and j+1 (j <= nb-2)
    double Wp[kRpl], Wm[kRpl], w_nm1 = 0.0;
#pragma unroll
    for (int r = 0; r < kRpl; r++) {
        const int j = row0 + r;
        Wp[r] = 0.0;
        Wm[r] = 0.0;
        if (j <= NB - 2) {
            const double Br = (r + 1 < kRpl) ? B[r + 1] : Bn;
            const double Cr = (r + 1 < kRpl) ? C[r + 1] : Cn;
            double w;
            face(B[r], Br, C[r], Cr, x[j], x[j + 1], Wp[r], Wm[r], w);
            if (j == NB - 2) w_nm1 = w;
        }
    }
    const double WpP = sup(Wp[kRpl - 1], 1), WmP = sup(Wm[kRpl - 1], 1);

    // rows a, b, c (cc_build_{left,interior,right}, Chang_Cooper.c:66-184)
    double A[kRpl], Bd[kRpl], Cc[kRpl];
#pragma unroll
    for (int r = 0; r < kRpl; r++) {
        const int m = row0 + r;
        const double k = dt / (1.0 * dx[m]);
        const double pB = (r > 0) ? B[r - 1] : Bp, pC = (r > 0) ? C[r - 1] : Cp;
        const double nB = (r + 1 < kRpl) ? B[r + 1] : Bn, nC = (r + 1 < kRpl) ? C[r + 1] : Cn;
        const double wpm = (r > 0) ? Wp[r - 1] : WpP, wmm = (r > 0) ? Wm[r - 1] : WmP;
        double av, bv, cv;
        if (m == 0) {
            if (fabs(C[r]) > 1.0e-200) {
                av = 0.0;
                bv = 1.0 + k * (0.0 + 0.5 * (C[r] + nC) / (x[1] - x[0]) * Wm[r]) + dT[r];
                cv = k * 0.5 * (C[r] + nC) / (x[1] - x[0]) * Wp[r];
            } else {
                av = 0.0;
                bv = 1.0 + k * 0.0 + dT[r];
                cv = k * 1.0 * 0.5 * (B[r] + nB);
            }
        } else if (m == NB - 1) {
            if (fabs(C[r]) > 1.0e-200) {
                av = k * (0.5 * (C[r] + pC)) / (x[m] - x[m - 1]) * wmm;
                bv = 1.0 + k * ((0.5 * (C[r] + pC)) / (x[m] - x[m - 1]) * wpm) + dT[r];
                if (isnan(av)) err |= kErrCcNan;
            } else {
                const double dlt = (fabs(pC) > 1.0e-200) ? face_delta(w_nm1) : 0.0;
                av = -dlt * 0.5 * (B[r] + pB) * dt / (1.0 * dx[m]);
                bv = 1.0 + k * (0.5 * (pB + B[r])) + dT[r];
            }
            cv = 0.0;
        } else if (fabs(C[r]) > 1.0e-200) {
            const double dxm_12 = x[m] - x[m - 1];
            const double dxm12 = x[m + 1] - x[m];
            const double cm_12 = 0.5 * (C[r] + pC);
            const double cm12 = 0.5 * (C[r] + nC);
            av = k * cm_12 / dxm_12 * wmm;
            bv = 1.0 + k * (cm_12 / dxm_12 * wpm + cm12 / dxm12 * Wm[r]) + dT[r];
            cv = k * cm12 / dxm12 * Wp[r];
        } else {
            const double bm_12 = 0.5 * (B[r] + pB);
            const double bm12 = 0.5 * (B[r] + nB);
            av = 0.0;
            bv = 1.0 + k * (1.0 * bm_12 - 0.0 * bm12) + dT[r];
            cv = k * 1.0 * bm12;
        }
        A[r] = av;
        Bd[r] = bv;
        Cc[r] = cv;
    }

    // ---- pivots: composed Moebius maps d -> b - a c_prev / d ----
    const double c_in = sup(Cc[kRpl - 1], 1);   // c of the row before this lane's first
    double t00 = 1.0, t01 = 0.0, t10 = 0.0, t11 = 1.0;
#pragma unroll
    for (int r = 0; r < kRpl; r++) {
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
    // incoming projective pivot (p, q) of this lane: exclusive prefix applied to (1, 0)
    double vp = sup(t00, 1), vq = sup(t10, 1);
    if (lane == 0) { vp = 1.0; vq = 0.0; }
    // cp of the previous row: -c_prev / d_prev with d_prev = vp / vq
    double cp_prev = (lane == 0) ? 0.0 : -c_in * vq / vp;
#pragma unroll
    for (int r = 0; r < kRpl; r++) {
        const int m = row0 + r;
        const double den = Bd[r] + A[r] * cp_prev;
        if (fabs(den) <= 1.0e-300) err |= kErrSingular;
        const double inv = 1.0 / den;
        F.inv[r] = inv;
        F.h[r] = A[r] * inv;
        F.q[r] = (m == NB - 1) ? 0.0 : Cc[r] * inv;
        F.sd[r] = src_dt[r] * inv;
        cp_prev = -Cc[r] * inv;
    }

    // ---- warp-scan multipliers of the two linear recurrences ----
    double H = 1.0, Q = 1.0;
#pragma unroll
    for (int r = 0; r < kRpl; r++) {
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
    return err;
}

// One implicit sub-step: N <- M^{-1} (N + dt src) with the factored M.
__device__ __forceinline__ void substep(const Factor &F, int lane, double N[kRpl])
{
    double y[kRpl];
    double acc = 0.0;
#pragma unroll
    for (int r = 0; r < kRpl; r++) {
        y[r] = fma(N[r], F.inv[r], F.sd[r]);
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
    for (int r = 0; r < kRpl; r++) {
        prev = fma(F.h[r], prev, y[r]);
        y[r] = prev;
    }
    acc = 0.0;
#pragma unroll
    for (int r = kRpl - 1; r >= 0; r--) acc = fma(F.q[r], acc, y[r]);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) {
        const int off = 1 << lv;
        const double o = sdn(acc, off);
        if (lane + off < 32) acc = fma(F.qk[lv], o, acc);
    }
    prev = sdn(acc, 1);
    if (lane == 31) prev = 0.0;
#pragma unroll
    for (int r = kRpl - 1; r >= 0; r--) {
        prev = fma(F.q[r], prev, y[r]);
        N[r] = prev;
    }
}

__global__ void __launch_bounds__(128) fused_slot_kernel(FusedParams P)
{
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const SnapArgs &a = P.a;
    const int t = gw >> 1, s = gw & 1;
    if (t >= a.ntracer) return;
    if (!(P.mp.species_mask & (1 << s))) return;
    const SegInfo g = seg_info(a.sched, t, P.slot, a.dt_snap);
    if (!g.active) return;
    const Bg bg = load_bg(a, t, g);
    const double tacc = segment_tacc(P.mp, a, g);
    const int dis = a.dis ? a.dis[t] : 0;
    SpeciesTerms T = make_species_terms(P.gt, s, bg, dis, a, g);
    const int row0 = lane * kRpl;

    double *Nrow = (s == 0 ? a.crp : a.cre) + (size_t)t * NB + row0;
    double N[kRpl];
#pragma unroll
    for (int r = 0; r < kRpl; r += 2) {
        const double2 v = *reinterpret_cast<const double2 *>(Nrow + r);
        N[r] = v.x;
        N[r + 1] = v.y;
    }
    const double *src = (s == 0) ? a.qpi : (P.inje ? P.inje : a.qepri);
    double sdt[kRpl];
#pragma unroll
    for (int r = 0; r < kRpl; r++) sdt[r] = src ? g.dt * src[(size_t)t * NB + row0 + r] : g.dt * 0.0;

    const DppForm on = dpp_form(P.mp, P.mp.dpp_model, bg, tacc);
    const double on_scale = (P.mp.dpp_model != kDppOff)
        ? eta_cap_scale(P.mp, P.gt, bg, a.mass ? a.mass[t] : 0.0, tacc, a.crp + (size_t)t * NB,
                        a.cre + (size_t)t * NB, 1)
        : 1.0;

    Factor F;
    int cur = -1;
    unsigned err = 0;
    for (int istep = 0; istep < g.steps; istep++) {
        const int want = (!g.windowed || (istep >= g.sl && istep < g.el)) ? 0 : 1;
        if (want != cur) {
            T.dform = want == 0 ? on : DppForm{0, 0.0};
            T.dpp_scale = want == 0 ? on_scale : 1.0;
            err |= factorize(T, sdt, lane, F);
            cur = want;
        }
        substep(F, lane, N);
    }
    if (err && lane == 0) atomicOr(a.err, err);
#pragma unroll
    for (int r = 0; r < kRpl; r += 2)
        *reinterpret_cast<double2 *>(Nrow + r) = make_double2(N[r], N[r + 1]);
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
        const SegInfo g = seg_info(a.sched, t, P.slot, a.dt_snap);
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

}  // namespace

int fused_reserve(Context &ctx, int cap)
{
    cudaFree(ctx.d_inje);
    ctx.d_inje = nullptr;
    CROMA_CUDA(cudaMalloc(&ctx.d_inje, (size_t)NB * cap * sizeof(double)));
    return 0;
}

int run_fused(Context &ctx, const SnapArgs &a)
{
    FusedParams P;
    P.a = a;
    P.gt = ctx.gt;
    P.mp = ctx.mp;
    P.np_min_qe = ctx.d_np_min_qe;
    const int nslots = ctx.mp.interp_max_segments < 1 ? 1 : ctx.mp.interp_max_segments;
    const int both = (ctx.mp.species_mask & 3) == 3;
    const long long nthreads = 2LL * a.ntracer * 32;
    const int blocks = (int)((nthreads + 127) / 128);
    for (int slot = 0; slot < nslots && slot < 64; slot++) {
        P.slot = slot;
        cudaEvent_t ev = nullptr;
        P.inje = nullptr;
        if (both) {
            dim3 sg((a.ntracer + 63) / 64, (NB + 63) / 64), sb(16, 16);
            timed_begin(ctx, kKindSecondary, &ev);
            fused_secondary_kernel<<<sg, sb, 0, ctx.stream>>>(P, ctx.d_inje);
            timed_end(ctx, kKindSecondary, ev);
            ctx.last_launches += 1;
            P.inje = ctx.d_inje;
        }
        timed_begin(ctx, kKindEvolve, &ev);
        fused_slot_kernel<<<blocks, 128, 0, ctx.stream>>>(P);
        timed_end(ctx, kKindEvolve, ev);
        ctx.last_launches += 1;
        CROMA_CUDA(cudaGetLastError());
    }
    return 0;
}

}  // namespace croma
