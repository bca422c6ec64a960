// plain.cu -- the plain FP64 evolve: the reference's data contract on a
// tracer-major, coalesced layout.
//
// For each coefficient-interpolation segment slot k (0 .. 15) three kernels
// run over every tracer whose snapshot has more than k segments:
//
//   plain_coeff_kernel   losses + Dpp + Chang-Cooper rows for one
//                        (tracer, species) per thread, written momentum-major
//                        [row][tracer] (tracer_fp_prepare_coeff_batches,
//                        src/tracer_fp_coef.c:218-359)
//   plain_secondary      secondary-electron source of the segment, a tiled
//                        [nb x nb] . [nb x tracers] product
//                        (prepare_secondary_sources_cell_major,
//                        src/fp_shared_core.c:1591-1672)
//   plain_steps_kernel   the segment's sub-steps, one Thomas system per thread
//                        with the reference's divides
//                        (tracer_fp_cpu_evolve, src/tracer_fp_cpu.c:149-190;
//                        fp_thomas_solve_ws, src/fp_shared_core.c:226-257)
//
// Segment timing follows tracer_fp_batch_execute_bucket
// (src/tracer_fp_batch.c:651-827): alpha = (k + 0.5) / nseg, split_range,
// the centred reacceleration window and the direct-t_acc schedule.
#include "croma_segment.cuh"

namespace croma {

namespace {

// Chang-Cooper rows of one system, streamed over the bins.  Sink(m, a, b, c).
// Rows follow cc_build_{interior,left,right} (Chang_Cooper.c:66-184) as
// assembled by fp_build_cc_coeffs_from_terms (fp_shared_core.c:660-704).
// The Chang-Cooper delta only enters rows whose diffusion coefficient is
// below 1e-200; there the reference's own zeroing leaves every delta it
// reads at 0 except delta[nm-1] of the right boundary, which is kept.
template <class Sink>
__device__ int cc_rows(const SpeciesTerms &T, Sink &sink)
{
    const SpeciesTables &st = T.gt->s[T.s];
    const double *x = st.p, *dx = st.dp;
    const double dt = T.dt;
    constexpr int nm = NB - 1;
    Terms t0 = T.at(0), t1 = T.at(1);
    double wp_prev, wm_prev, w_prev;
    face(t0.B, t1.B, t0.C, t1.C, x[0], x[1], wp_prev, wm_prev, w_prev);
    {   // left boundary
        const double k = dt / (1.0 * dx[0]);
        double a, b, c;
        if (fabs(t0.C) > 1.0e-200) {
            a = 0.0;
            b = 1.0 + k * (0.0 + 0.5 * (t0.C + t1.C) / (x[1] - x[0]) * wm_prev) + t0.dtT;
            c = k * 0.5 * (t0.C + t1.C) / (x[1] - x[0]) * wp_prev;
        } else {
            a = 0.0;
            b = 1.0 + k * 0.0 + t0.dtT;
            c = k * 1.0 * 0.5 * (t0.B + t1.B);
        }
        sink(0, a, b, c);
    }
    Terms prev = t0, cur = t1;
    for (int m = 1; m < nm; m++) {
        const Terms next = T.at(m + 1);
        double wp_cur, wm_cur, w_cur;
        face(cur.B, next.B, cur.C, next.C, x[m], x[m + 1], wp_cur, wm_cur, w_cur);
        const double k = dt / (1.0 * dx[m]);
        double a, b, c;
        if (fabs(cur.C) > 1.0e-200) {
            const double dxm_12 = x[m] - x[m - 1];
            const double dxm12 = x[m + 1] - x[m];
            const double cm_12 = 0.5 * (cur.C + prev.C);
            const double cm12 = 0.5 * (cur.C + next.C);
            a = k * cm_12 / dxm_12 * wm_prev;
            b = 1.0 + k * (cm_12 / dxm_12 * wp_prev + cm12 / dxm12 * wm_cur) + cur.dtT;
            c = k * cm12 / dxm12 * wp_cur;
        } else {
            const double bm_12 = 0.5 * (cur.B + prev.B);
            const double bm12 = 0.5 * (cur.B + next.B);
            a = 0.0;
            b = 1.0 + k * (1.0 * bm_12 - 0.0 * bm12) + cur.dtT;
            c = k * 1.0 * bm12;
        }
        sink(m, a, b, c);
        prev = cur;
        cur = next;
        wp_prev = wp_cur;
        wm_prev = wm_cur;
        w_prev = w_cur;
    }
    {   // right boundary (m = nm): prev = nm-1, cur = nm
        const double k = dt / (1.0 * dx[nm]);
        double a, b;
        if (fabs(cur.C) > 1.0e-200) {
            a = k * (0.5 * (cur.C + prev.C)) / (x[nm] - x[nm - 1]) * wm_prev;
            b = 1.0 + k * ((0.5 * (cur.C + prev.C)) / (x[nm] - x[nm - 1]) * wp_prev) + cur.dtT;
            if (isnan(a)) return -1;
        } else {
            const double dlt = (fabs(prev.C) > 1.0e-200) ? face_delta(w_prev) : 0.0;
            a = -dlt * 0.5 * (cur.B + prev.B) * dt / (1.0 * dx[nm]);
            b = 1.0 + k * (0.5 * (prev.B + cur.B)) + cur.dtT;
        }
        sink(nm, a, b, 0.0);
    }
    return 0;
}

struct PlainParams {
    SnapArgs a;
    GridTables gt;
    ModelParams mp;
    int slot;
    int cap;
    int need_off;
    double *coef;        // [set][species][3][NB][cap]
    double *seg_ngas;    // [cap]
};

__device__ __forceinline__ double *coef_ptr(const PlainParams &P, int set, int s, int k)
{
    return P.coef + ((size_t)((set * 2 + s) * 3 + k) * NB) * (size_t)P.cap;
}

struct GlobalSink {
    double *a, *b, *c;
    size_t stride;
    int t;
    __device__ void operator()(int m, double av, double bv, double cv)
    {
        a[m * stride + t] = av;
        b[m * stride + t] = bv;
        c[m * stride + t] = cv;
    }
};

__global__ void __launch_bounds__(128) plain_coeff_kernel(PlainParams P)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;   // 0 proton, 1 electron
    const SnapArgs &a = P.a;
    if (t >= a.ntracer) return;
    if (!(P.mp.species_mask & (1 << s))) return;
    const SegInfo g = seg_info(a.sched, t, P.slot, a.dt_snap);
    if (!g.active) return;
    const Bg bg = load_bg(a, t, g);
    if (s == 0) P.seg_ngas[t] = bg.n_gas;

    const double tacc = segment_tacc(P.mp, a, g);
    const int dis = a.dis ? a.dis[t] : 0;
    SpeciesTerms T = make_species_terms(P.gt, s, bg, dis, a, g);

    // The ghost-edge loss and diffusion terms only reach the rows through
    // the left ghost face, whose weights multiply a zero flux there
    // (c_12 = 0, Chang_Cooper.c:125-131), so they are not formed.

    const size_t stride = (size_t)P.cap;
    for (int set = 0; set < (P.need_off && g.windowed ? 2 : 1); set++) {
        if (set == 0) {
            T.dform = dpp_form(P.mp, P.mp.dpp_model, bg, tacc);
            T.dpp_scale = (P.mp.dpp_model != kDppOff)
                ? eta_cap_scale(P.mp, P.gt, bg, a.mass ? a.mass[t] : 0.0, tacc, a.crp + t, a.cre + t, stride)
                : 1.0;
        } else {
            T.dform = DppForm{0, 0.0};
            T.dpp_scale = 1.0;
        }
        GlobalSink sink{coef_ptr(P, set, s, 0), coef_ptr(P, set, s, 1), coef_ptr(P, set, s, 2), stride, t};
        if (cc_rows(T, sink) != 0) atomicOr(a.err, kErrCcNan);
    }
}

// Secondary source of the segment: inje[je][t] = Gyr n_gas sum_jp N_p[jp][t] fqe[jp][je] + qepri.
// 64 x 64 output tile per block, 16 x 16 threads, 4 x 4 outputs each;
// the proton index runs upward from fqe_jp0 as in the reference.
__global__ void __launch_bounds__(256) plain_secondary_kernel(PlainParams P, double *inje)
{
    __shared__ double sF[16][64];
    __shared__ double sN[16][64];
    const SnapArgs &a = P.a;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int t0 = blockIdx.x * 64, je0 = blockIdx.y * 64;
    const size_t stride = (size_t)P.cap;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
    const int tid = ty * 16 + tx;
    for (int jp0 = P.gt.fqe_jp0; jp0 < NB; jp0 += 16) {
        for (int q = tid; q < 16 * 64; q += 256) {
            const int r = q / 64, col = q % 64;
            const int jp = jp0 + r;
            sF[r][col] = (jp < NB && je0 + col < NB) ? P.gt.fqe[(size_t)jp * NB + je0 + col] : 0.0;
            const int t = t0 + col;
            sN[r][col] = (jp < NB && t < a.ntracer) ? a.crp[(size_t)jp * stride + t] : 0.0;
        }
        __syncthreads();
        const int kmax = (NB - jp0) < 16 ? (NB - jp0) : 16;
        for (int r = 0; r < kmax; r++) {
            double f[4], n[4];
#pragma unroll
            for (int i = 0; i < 4; i++) f[i] = sF[r][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) n[j] = sN[r][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] += n[j] * f[i];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int je = je0 + ty + 16 * i;
        if (je >= NB) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int t = t0 + tx + 16 * j;
            if (t >= a.ntracer) continue;
            const SegInfo g = seg_info(a.sched, t, P.slot, a.dt_snap);
            if (!g.active) continue;
            const double q = a.qepri ? a.qepri[(size_t)je * stride + t] : 0.0;
            inje[(size_t)je * stride + t] = acc[i][j] * kGyr * P.seg_ngas[t] + q;
        }
    }
}

__global__ void __launch_bounds__(128) plain_steps_kernel(PlainParams P, const double *inje)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    const SnapArgs &a = P.a;
    if (t >= a.ntracer) return;
    if (!(P.mp.species_mask & (1 << s))) return;
    const SegInfo g = seg_info(a.sched, t, P.slot, a.dt_snap);
    if (!g.active) return;
    const size_t stride = (size_t)P.cap;
    double *N = (s == 0 ? a.crp : a.cre) + t;
    const double *src = (s == 0) ? a.qpi : (inje ? inje : a.qepri);
    if (src) src += t;
    double cp[NB];
    for (int istep = 0; istep < g.steps; istep++) {
        const int use_on = !g.windowed || (istep >= g.sl && istep < g.el);
        const int set = use_on ? 0 : 1;
        const double *A = coef_ptr(P, set, s, 0) + t;
        const double *B = coef_ptr(P, set, s, 1) + t;
        const double *Cc = coef_ptr(P, set, s, 2) + t;
        double b0 = B[0];
        if (fabs(b0) <= 1.0e-300) { atomicOr(a.err, kErrSingular); return; }
        cp[0] = -Cc[0] / b0;
        double xprev = ((src ? g.dt * src[0] : g.dt * 0.0) + N[0]) / b0;
        N[0] = xprev;
        for (int i = 1; i < NB; i++) {
            const size_t o = (size_t)i * stride;
            const double ai = A[o];
            const double den = B[o] + ai * cp[i - 1];
            if (fabs(den) <= 1.0e-300) { atomicOr(a.err, kErrSingular); return; }
            cp[i] = (i == NB - 1) ? 0.0 : -Cc[o] / den;
            const double r = (src ? g.dt * src[o] : g.dt * 0.0) + N[o];
            xprev = (r + ai * xprev) / den;
            N[o] = xprev;
        }
        double xnext = N[(size_t)(NB - 1) * stride];
        for (int i = NB - 2; i >= 0; i--) {
            const size_t o = (size_t)i * stride;
            const double x = N[o] - cp[i] * xnext;
            N[o] = x;
            xnext = x;
        }
    }
}

__global__ void transpose_kernel(const double *in, double *out, int rows, int cols)
{
    // in [rows][cols] -> out [cols][rows]
    __shared__ double tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[i][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[threadIdx.x][i];
    }
}

}  // namespace

int plain_reserve(Context &ctx, int cap)
{
    cudaFree(ctx.d_coef);
    cudaFree(ctx.d_inje);
    cudaFree(ctx.d_seg_ngas);
    ctx.d_coef = ctx.d_inje = ctx.d_seg_ngas = nullptr;
    const int sets = ctx.mp.window_centred ? 2 : 1;
    CROMA_CUDA(cudaMalloc(&ctx.d_coef, (size_t)sets * 2 * 3 * NB * (size_t)cap * sizeof(double)));
    CROMA_CUDA(cudaMalloc(&ctx.d_inje, (size_t)NB * cap * sizeof(double)));
    CROMA_CUDA(cudaMalloc(&ctx.d_seg_ngas, (size_t)cap * sizeof(double)));
    return 0;
}

int run_plain(Context &ctx, const SnapArgs &a)
{
    PlainParams P;
    P.a = a;
    P.gt = ctx.gt;
    P.mp = ctx.mp;
    P.cap = ctx.cap;
    P.need_off = ctx.mp.window_centred;
    P.coef = ctx.d_coef;
    P.seg_ngas = ctx.d_seg_ngas;
    const int nslots = ctx.mp.interp_max_segments < 1 ? 1 : ctx.mp.interp_max_segments;
    const int protons = ctx.mp.species_mask & CROMA_SPECIES_PROTON;
    const int electrons = ctx.mp.species_mask & CROMA_SPECIES_ELECTRON;
    const dim3 blk(128), grd((a.ntracer + 127) / 128, 2);
    for (int slot = 0; slot < nslots && slot < 64; slot++) {
        P.slot = slot;
        cudaEvent_t ev = nullptr;
        timed_begin(ctx, kKindCoeff, &ev);
        plain_coeff_kernel<<<grd, blk, 0, ctx.stream>>>(P);
        timed_end(ctx, kKindCoeff, ev);
        ctx.last_launches += 1;
        const double *inje = nullptr;
        if (protons && electrons) {
            dim3 sg((a.ntracer + 63) / 64, (NB + 63) / 64), sb(16, 16);
            timed_begin(ctx, kKindSecondary, &ev);
            plain_secondary_kernel<<<sg, sb, 0, ctx.stream>>>(P, ctx.d_inje);
            timed_end(ctx, kKindSecondary, ev);
            ctx.last_launches += 1;
            inje = ctx.d_inje;
        }
        timed_begin(ctx, kKindEvolve, &ev);
        plain_steps_kernel<<<grd, blk, 0, ctx.stream>>>(P, inje);
        timed_end(ctx, kKindEvolve, ev);
        ctx.last_launches += 1;
        CROMA_CUDA(cudaGetLastError());
    }
    return 0;
}

int transpose_to_device(Context &ctx, const double *h_cell_major, double *d_mom_major, int n)
{
    // host [n][NB] -> staging -> device [NB][cap]
    double *stg = ctx.d_layout_tmp;
    CROMA_CUDA(cudaMemcpyAsync(stg, h_cell_major, (size_t)n * NB * sizeof(double),
                               cudaMemcpyHostToDevice, ctx.stream));
    if (n == ctx.cap) {
        transpose_kernel<<<dim3(NB / 32, (n + 31) / 32), dim3(32, 8), 0, ctx.stream>>>(stg, d_mom_major, n, NB);
    } else {
        return -1;
    }
    CROMA_CUDA(cudaGetLastError());
    return 0;
}

int transpose_to_host(Context &ctx, const double *d_mom_major, double *h_cell_major, int n)
{
    double *stg = ctx.d_layout_tmp;
    if (n != ctx.cap) return -1;
    transpose_kernel<<<dim3((n + 31) / 32, NB / 32), dim3(32, 8), 0, ctx.stream>>>(d_mom_major, stg, NB, n);
    CROMA_CUDA(cudaGetLastError());
    CROMA_CUDA(cudaMemcpyAsync(h_cell_major, stg, (size_t)n * NB * sizeof(double),
                               cudaMemcpyDeviceToHost, ctx.stream));
    return 0;
}

}  // namespace croma
