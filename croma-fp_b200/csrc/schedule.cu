// schedule.cu -- per-snapshot sub-step schedule on the device.
//
// Compiled with --fmad=false: the sub-step count is an integer decision
// (ceil of a quotient, a quantisation ladder) taken on floating-point loss
// rates, and the reference takes it with separately rounded multiplies and
// adds.  Keeping the same rounding sequence here makes nsub / n_on
// reproduce the reference's integers.
//
//   endpoint losses   tracer_fp_prepare_nsub_loss_endpoints, src/tracer_fp_nsub.c:242-282
//   nsub / n_on       compute_nsubsteps_core, src/tracer_fp_nsub.c:94-187
//   ladder            quantize_dt_sub / quantize_on_fraction, src/tracer_fp_nsub.c:37-92
//   segments          tracer_fp_choose_coeff_interp_segments, src/tracer_fp_setup.c:73-95
//   buckets           tracer_bucket_build_snapshot, src/tracer_fp_bucket.c:208-262
#include <cub/cub.cuh>

#include "croma_ctx.cuh"

namespace croma {

namespace {

__device__ double quantize_dt_sub(double t)
{
    const double ladder[10] = {1.0, 1.25, 1.6, 2.0, 2.5, 3.2, 4.0, 5.0, 6.4, 8.0};
    if (!(t > 0.0) || !isfinite(t)) return t;
    const double e10 = floor(log10(t));
    const double scale = pow(10.0, e10);
    const double norm = t / scale;
    double chosen = ladder[0];
    for (int i = 0; i < 10; i++) {
        if (ladder[i] <= norm) chosen = ladder[i];
        else break;
    }
    return chosen * scale;
}

__device__ double quantize_on_fraction(double f)
{
    const double bins[5] = {1.0 / 8.0, 1.0 / 4.0, 1.0 / 3.0, 1.0 / 2.0, 1.0};
    if (!(f > 0.0) || !isfinite(f)) return 1.0;
    if (f >= 1.0) return 1.0;
    double chosen = bins[0], best = fabs(f - chosen);
    for (int i = 1; i < 5; i++) {
        const double d = fabs(f - bins[i]);
        if (d < best) { chosen = bins[i]; best = d; }
    }
    return chosen;
}

__device__ int coeff_segments(const ModelParams &mp, int nsub, int allow)
{
    int seg = 1;
    int max_seg = mp.interp_max_segments;
    if (!allow || nsub <= 1) return 1;
    if (mp.interp_min_steps <= 0) return 1;
    if (max_seg < 1) max_seg = 1;
    const int max_allowed = nsub / mp.interp_min_steps;
    if (max_allowed < 1) return 1;
    while (seg <= 1073741823 && seg * 2 <= max_seg && seg * 2 <= max_allowed) seg *= 2;
    if (seg > nsub) seg = nsub;
    if (seg < 1) seg = 1;
    return seg;
}

__global__ void nsub_kernel(ModelParams mp, int ntracer, const double *bg, const double *ic_row,
                            double p_lo, double p_hi, double pe_lo, double pe_hi,
                            double dt_snap, int allow, Schedule s)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntracer) return;
    const double ng = bg[0 * (size_t)ntracer + t];
    const double kbt = bg[1 * (size_t)ntracer + t];
    const double bf = bg[2 * (size_t)ntracer + t];
    const double dvv = bg[3 * (size_t)ntracer + t];
    const double lt = bg[4 * (size_t)ntracer + t];
    const double dv = bg[5 * (size_t)ntracer + t];

    const double rp_lo = coulomb_p_from_p(ng, p_lo, kbt) + 1.0 / 3.0 * dvv * p_lo;
    const double rp_hi = coulomb_p_from_p(ng, p_hi, kbt) + 1.0 / 3.0 * dvv * p_hi;
    const double re_lo = b_synch(pe_lo, bf) + ic_row[0] + b_coulomb_e(ng, pe_lo) + 1.0 / 3.0 * dvv * pe_lo;
    const double re_hi = b_synch(pe_hi, bf) + ic_row[NB - 1] + b_coulomb_e(ng, pe_hi) + 1.0 / 3.0 * dvv * pe_hi;

    const double te0 = pe_lo / re_lo;
    const double tp0 = p_lo / rp_lo;
    const double teN = pe_hi / re_hi;
    const double tpN = p_hi / rp_hi;
    const double tmin = fmin(fabs(tp0), fmin(fabs(teN), fmin(fabs(te0), fabs(tpN))));

    double target = dt_snap / 10.0;
    if (isfinite(tmin) && tmin > 0.0) {
        const double stab = mp.nsub_safety * tmin;
        if (stab < target) target = stab;
    }
    if (target <= 0.0 || !isfinite(target)) target = dt_snap / 10.0;
    double tn = ceil(dt_snap / target);
    if (!isfinite(tn) || tn > 1000000.0) tn = 1000000.0;
    if (tn < 10.0) tn = 10.0;
    double used = quantize_dt_sub(target);
    if (!(used > 0.0) || !isfinite(used) || used > target) used = target;
    double raw = ceil(dt_snap / used);
    if (!isfinite(raw) || raw > 1000000.0) raw = 1000000.0;
    if (raw < 10.0) raw = 10.0;
    int nsub = (int)raw;
    unsigned char capped = 0;
    if (mp.nsub_max > 0 && nsub > mp.nsub_max) {
        nsub = mp.nsub_max;
        capped = 1;
    }
    double onf = 1.0;
    if (mp.window_centred && mp.f_eddy > 0.0 && dv > 0.0) {
        const double t_eddy = lt * 3.0857e24 / dv / 3.1536e16;
        if (mp.f_eddy * t_eddy < dt_snap) onf = quantize_on_fraction(mp.f_eddy * t_eddy / dt_snap);
    }
    int non = (int)floor((double)nsub * onf + 0.5);
    if (non < 1) non = 1;
    if (non > nsub) non = nsub;

    s.nsub[t] = nsub;
    s.non[t] = non;
    s.target[t] = (int)tn;
    s.capped[t] = capped;
    s.nseg[t] = coeff_segments(mp, nsub, allow);
}

// ---- bucket build: first-appearance order of the (nsub, n_on) key ----
__global__ void make_keys_kernel(int n, const int *nsub, const int *non, unsigned long long *keys,
                                 int *vals)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    keys[t] = ((unsigned long long)(unsigned)nsub[t] << 32) | (unsigned)non[t];
    vals[t] = t;
}

// After a stable sort by key: head flags -> segment index per element.
__global__ void seg_heads_kernel(int n, const unsigned long long *keys, int *head)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// seg_of[i] = inclusive-scan(head)[i] - 1.  For segment heads, record
// (first tracer, segment) pairs keyed by the first tracer index.
__global__ void seg_first_kernel(int n, const int *seg_incl, const int *sorted_t,
                                 unsigned long long *first_keys, int *first_seg)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int seg = seg_incl[i] - 1;
    if (i == 0 || seg_incl[i] != seg_incl[i - 1]) {
        first_keys[seg] = (unsigned long long)sorted_t[i];
        first_seg[seg] = seg;
    }
}

// bucket_of_seg[seg] = rank of the segment's first tracer (ranks beyond
// the segment count belong to the all-ones padding and are skipped).
__global__ void seg_rank_kernel(int n, const int *nseg_dev, const int *seg_by_first,
                                int *bucket_of_seg)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n || r >= *nseg_dev) return;
    bucket_of_seg[seg_by_first[r]] = r;
}

__global__ void assign_bucket_kernel(int n, const int *seg_incl, const int *sorted_t,
                                     const int *bucket_of_seg, int *bucket_ids, int *bucket_count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = bucket_of_seg[seg_incl[i] - 1];
    bucket_ids[sorted_t[i]] = b;
    atomicAdd(&bucket_count[b], 1);
}

// Members listed bucket by bucket in ascending tracer order: a stable
// pass over tracers in index order within each bucket is a stable sort
// of (bucket, tracer) by bucket, which the radix sort below provides.
__global__ void bucket_keys_kernel(int n, const int *bucket_ids, unsigned long long *keys, int *vals)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    keys[t] = (unsigned long long)(unsigned)bucket_ids[t];
    vals[t] = t;
}

}  // namespace

int schedule_reserve(Context &ctx, int cap)
{
    // ints: nsub, non, target, nseg, bucket_ids, bucket_indices, nbuckets(+pad), and aux
    if (ctx.d_sched_int) {
        dev_free(ctx, ctx.d_sched_int);
        dev_free(ctx, ctx.d_capped);
        dev_free(ctx, ctx.d_cub_tmp);
        dev_free(ctx, ctx.d_keys);
        dev_free(ctx, ctx.d_vals);
        ctx.d_sched_int = nullptr;
    }
    const size_t n = (size_t)cap;
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_sched_int, (n * 6 + 32) * sizeof(int)));
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_capped, n));
    int *p = ctx.d_sched_int;
    ctx.sched.nsub = p;
    ctx.sched.non = p + n;
    ctx.sched.target = p + 2 * n;
    ctx.sched.nseg = p + 3 * n;
    ctx.sched.bucket_ids = p + 4 * n;
    ctx.sched.bucket_indices = p + 5 * n;
    ctx.sched.nbuckets = p + 6 * n;
    ctx.sched.capped = ctx.d_capped;
    // keys/vals double buffers + aux (head/scan, first keys, seg ids, bucket_of_seg, counts)
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_keys, n * 3 * sizeof(unsigned long long)));
    ctx.d_keys_alt = ctx.d_keys + n;
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_vals, n * 8 * sizeof(int)));
    ctx.d_vals_alt = ctx.d_vals + n;
    ctx.d_seg_aux = ctx.d_vals + 2 * n;
    size_t b1 = 0, b2 = 0;
    cub::DoubleBuffer<unsigned long long> kb(ctx.d_keys, ctx.d_keys_alt);
    cub::DoubleBuffer<int> vb(ctx.d_vals, ctx.d_vals_alt);
    CROMA_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b1, kb, vb, cap, 0, 64, ctx.stream));
    CROMA_CUDA(cub::DeviceScan::InclusiveSum(nullptr, b2, ctx.d_seg_aux, ctx.d_seg_aux, cap, ctx.stream));
    ctx.cub_tmp_bytes = (b1 > b2 ? b1 : b2) + 256;
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_cub_tmp, ctx.cub_tmp_bytes));
    return 0;
}

int run_schedule(Context &ctx, const SnapArgs &a)
{
    const int n = a.ntracer;
    const int blk = 256, grd = (n + blk - 1) / blk;
    nsub_kernel<<<grd, blk, 0, ctx.stream>>>(ctx.mp, n, a.bg_curr, a.ic_curr, ctx.h_p[0][0],
                                             ctx.h_p[0][NB - 1], ctx.h_p[1][0], ctx.h_p[1][NB - 1],
                                             a.dt_snap, a.allow_interp, a.sched);
    CROMA_CUDA(cudaGetLastError());
    ctx.last_launches += 1;

    // ---- bucket build ----
    const size_t N = (size_t)n;
    int *head = ctx.d_seg_aux;              // [n] head flags, scanned in place
    int *first_seg = ctx.d_seg_aux + N;     // [n]
    int *bucket_of_seg = ctx.d_seg_aux + 2 * N;
    int *seg_by_first = ctx.d_seg_aux + 3 * N;
    int *counts = ctx.d_seg_aux + 4 * N;
    unsigned long long *first_keys = ctx.d_keys + 2 * N;
    size_t tmp = ctx.cub_tmp_bytes;

    make_keys_kernel<<<grd, blk, 0, ctx.stream>>>(n, a.sched.nsub, a.sched.non, ctx.d_keys, ctx.d_vals);
    cub::DoubleBuffer<unsigned long long> kb(ctx.d_keys, ctx.d_keys_alt);
    cub::DoubleBuffer<int> vb(ctx.d_vals, ctx.d_vals_alt);
    CROMA_CUDA(cub::DeviceRadixSort::SortPairs(ctx.d_cub_tmp, tmp, kb, vb, n, 0, 64, ctx.stream));
    const unsigned long long *skeys = kb.Current();
    const int *sorted_t = vb.Current();
    seg_heads_kernel<<<grd, blk, 0, ctx.stream>>>(n, skeys, head);
    tmp = ctx.cub_tmp_bytes;
    CROMA_CUDA(cub::DeviceScan::InclusiveSum(ctx.d_cub_tmp, tmp, head, head, n, ctx.stream));
    // sorted_t lives in one of the two value buffers; keep it intact while the
    // segment-first pairs are sorted through the other key buffer and aux ints.
    // (first tracer, segment) pairs; unused tail entries carry all-ones keys
    // so that they sort last.
    CROMA_CUDA(cudaMemsetAsync(first_keys, 0xFF, N * sizeof(unsigned long long), ctx.stream));
    seg_first_kernel<<<grd, blk, 0, ctx.stream>>>(n, head, sorted_t, first_keys, first_seg);
    {
        unsigned long long *fk_alt = (kb.Current() == ctx.d_keys) ? ctx.d_keys_alt : ctx.d_keys;
        cub::DoubleBuffer<unsigned long long> fkb(first_keys, fk_alt);
        cub::DoubleBuffer<int> fvb(first_seg, seg_by_first);
        tmp = ctx.cub_tmp_bytes;
        CROMA_CUDA(cub::DeviceRadixSort::SortPairs(ctx.d_cub_tmp, tmp, fkb, fvb, n, 0, 32, ctx.stream));
        seg_rank_kernel<<<grd, blk, 0, ctx.stream>>>(n, head + (n - 1), fvb.Current(), bucket_of_seg);
        CROMA_CUDA(cudaMemsetAsync(counts, 0, N * sizeof(int), ctx.stream));
        assign_bucket_kernel<<<grd, blk, 0, ctx.stream>>>(n, head, sorted_t, bucket_of_seg,
                                                          a.sched.bucket_ids, counts);
        CROMA_CUDA(cudaMemcpyAsync(a.sched.nbuckets, head + (n - 1), sizeof(int),
                                   cudaMemcpyDeviceToDevice, ctx.stream));
    }
    CROMA_CUDA(cudaGetLastError());
    ctx.last_launches += 6;

    // member lists: stable sort of (bucket id, tracer) by bucket id
    {
        unsigned long long *k0 = ctx.d_keys, *k1 = ctx.d_keys_alt;
        int *v0 = ctx.d_vals, *v1 = ctx.d_vals_alt;
        bucket_keys_kernel<<<grd, blk, 0, ctx.stream>>>(n, a.sched.bucket_ids, k0, v0);
        cub::DoubleBuffer<unsigned long long> bkb(k0, k1);
        cub::DoubleBuffer<int> bvb(v0, v1);
        tmp = ctx.cub_tmp_bytes;
        CROMA_CUDA(cub::DeviceRadixSort::SortPairs(ctx.d_cub_tmp, tmp, bkb, bvb, n, 0, 32, ctx.stream));
        CROMA_CUDA(cudaMemcpyAsync(a.sched.bucket_indices, bvb.Current(), N * sizeof(int),
                                   cudaMemcpyDeviceToDevice, ctx.stream));
    }
    CROMA_CUDA(cudaGetLastError());
    ctx.last_launches += 6;
    return 0;
}

}  // namespace croma
