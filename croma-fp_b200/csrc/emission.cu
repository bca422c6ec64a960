// emission.cu -- the kernel tables of the emission integrals, built on the
// device, and the per-snapshot emissivities of a context's resident spectra
// written straight to device memory.
//
// Tables (the reference builds them on the host, once per run or, for IC,
// per emitted snapshot):
//   synchrotron F(x) = x int_x^inf K_5/3     SYN_logFx_table, src/Synchrotron.c:31-41
//                                            (the reference calls GNU GSL's
//                                            gsl_sf_synchrotron_1 for x <= 300)
//   synchrotron pitch-kernel table           tracer_fp_synch_data_init_tables +
//                                            tracer_fp_refresh_synch_kernel_table,
//                                            src/tracer_fp_synch.c:87-121, 175-240
//   hadronic gamma / neutrino kernels        prepare_gamma/neutrino_kernel_flat,
//                                            src/fp_shared_core.c:1724-1778
//   inverse-Compton kernel at redshift z     prepare_ic_kernel_flat,
//                                            src/fp_shared_core.c:1780-1807
//
// Per snapshot (croma_b200_emission_run), from the spectra the snapshot
// starts from (include/tracer_fp_solve.inc:117-426 emits before the solve):
//   IC, gamma, neutrino: one FP64 tensor-core GEMM per kind,
//     eps[t][k] = s_t sum_j N[t][j] W[j][k],
//   with the bin weights of the reference's sums folded into W (dp for IC;
//   the trapezoid of Q_one, src/EMISSION.c:297-308, with beta_p and E_k / 2
//   for the hadronic kinds) and s_t = n_gas of the tracer (1 for IC);
//   synchrotron: one warp per tracer, the log-K interpolation of
//   prepare_synch_emission_cell_major (src/fp_shared_core.c:2070-2112,
//   tracer_fp_interp_synch_kernel_logk :2054-2068) over tables of K and
//   log K, the bins split over the lanes, bins from 2 up to the first je
//   whose N[je+1] is not positive; b_dyn = B of the snapshot's background
//   (field 2), logb = log10(B / 1e-6 G) with a non-positive or non-finite B
//   taken as 1e-30 (tracer_fp_logb_range_from_snapshot,
//   src/tracer_fp_synch.c:123-152).  Tracers run sorted by their log-B
//   plane so that a block shares each table row through shared memory.
// The sums run in a different order from the reference's sequential loops:
// the results agree to rounding, not bit for bit.
#include <cstdio>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

#define np CROMA_NB
#define npe CROMA_NB
#include "../../include/fp_cuda_backend.h"
#include "croma_emission.cuh"
#include "croma_hadronic.cuh"

namespace croma {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// Synchrotron F(x).  With K_nu(s) = int_0^inf exp(-s cosh t) cosh(nu t) dt the
// s-integral has the closed form int_x^inf exp(-s cosh t) ds = exp(-x cosh t) /
// cosh t, so
//     F(x) = x int_0^inf exp(-x cosh t) cosh(5t/3) / cosh(t) dt.
// The integrand is even and analytic in a strip about the real axis and
// decays double-exponentially, so the trapezoid rule converges geometrically
// in the step: h = 1/32 agrees with a multiprecision evaluation to ~1e-14
// for every x of the table.  The range stops where x cosh t = 800 (the
// integrand is below the smallest double there).  For x > 300 the reference
// itself uses the asymptotic form sqrt(pi/2) exp(-x) sqrt(x), kept here.
constexpr double kFxStep = 1.0 / 32.0;

__device__ __forceinline__ double fx_integrand(double x, double t)
{
    const double e = exp(t), e53 = exp(t * (5.0 / 3.0));
    const double ch = 0.5 * (e + 1.0 / e), ch53 = 0.5 * (e53 + 1.0 / e53);
    return exp(-x * ch) * (ch53 / ch);
}

// log10 F at each logx, one warp per abscissa (lanes stride the trapezoid
// nodes, a shuffle tree sums them).
__global__ void __launch_bounds__(256) synch_logfx_kernel(int nx, const double *logx, double *logfx)
{
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (i >= nx) return;
    const double x = pow(10.0, logx[i]);
    double F;
    if (x > 300.0) {
        F = sqrt(0.5 * kPi) * exp(-x) * pow(x, 0.5);
    } else {
        const double r = fmax(2.0, 800.0 / x);
        const double tmax = log(r + sqrt(r * r - 1.0));
        const int n = (int)ceil(tmax / kFxStep);
        double s = 0.0;
        for (int k = 1 + lane; k <= n; k += 32) s += fx_integrand(x, k * kFxStep);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(kFull, s, off);
        s += 0.5 * exp(-x);   // t = 0: exp(-x) cosh 0 / cosh 0, half weight
        F = x * kFxStep * s;
    }
    if (lane == 0) logfx[i] = log10(F);
}

// ---------------------------------------------------------------------------
// Kernel tables, one thread per (band, momentum bin).
__global__ void gamma_table_kernel(int nbins, const double *E, const double *p, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbins * NB) return;
    out[i] = gamma_kernel(E[i / NB], p[i % NB]);
}

__global__ void neutrino_table_kernel(int nbins, const double *E, const double *p, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbins * NB) return;
    out[i] = neutrino_kernel(E[i / NB], p[i % NB]);
}

__global__ void ic_table_kernel(IcConsts k, int nbins, const double *nu, const double *p, double z, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbins * NB) return;
    const double pe = p[i % NB];
    out[i] = ic_emissivity(k, nu[i / NB], sqrt(1.0 + pe * pe), z);
}

// logy[nf][je][k] = log10(nu_nf / (1e-6 nu_crit[je][k])), nu_crit the
// critical frequency at B = 1 (SYN_nu_crit_subB / SYN_crit_freq /
// SYN_logy_table, src/Synchrotron.c:9-51).
__global__ void synch_logy_kernel(int nfreq, int ntheta, const double *nus, const double *p, const double *theta,
                                  double *logy)
{
    const long long total = (long long)nfreq * NB * ntheta;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i % ntheta);
        const long long r = i / ntheta;
        const int je = (int)(r % NB), nf = (int)(r / NB);
        const double gamma2 = 1.0 + pow(p[je], 2.0);
        const double nu_crit = 1.0 * gamma2 * 4.194284e+06 * sin(theta[k]);
        logy[i] = log10(nus[nf] / (1.0e-6 * nu_crit));
    }
}

// log K of the pitch-kernel table where K > 0, NaN where it is not: the
// interpolation takes the log form only when both ends are positive, so a
// NaN end sends it to the linear form on K itself.
__global__ void log_table_kernel(long long n, const double *K, double *logK)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = K[i];
        logK[i] = (v > 0.0) ? log(v) : __longlong_as_double(0x7ff8000000000000LL);
    }
}

// ---------------------------------------------------------------------------
// Emissivity GEMM: out[t][k] = scale[t] * sum_j N[t][j] W[j][k] for k < ncols,
// N the resident spectra [ntracer][NB], W [NB][wpitch] (zero past ncols).
// FP64 tensor cores (mma.sync m8n8k4 .f64); 128 x 64 output tile per 256
// threads, each warp 32 x 32 as 4 x 4 fragments; k-tiles of 16 double-buffered
// in shared memory by cp.async.  Row pitches 20 and 68 doubles keep the
// fragment reads of a half warp on distinct bank pairs.
constexpr int kEM = 128, kEN = 64, kEK = 16;
constexpr int kEPitchA = kEK + 4, kEPitchB = kEN + 4;

struct EmisGemmSmem {
    double A[2][kEM][kEPitchA];
    double B[2][kEK][kEPitchB];
};

__device__ __forceinline__ void cp16(void *dst, const void *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}

__device__ __forceinline__ void mma_f64(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256, 2) emission_gemm_kernel(int nrows, int ncols, int wpitch, const double *N,
                                                               const double *W, const double *scale,
                                                               int scale_stride, double *out)
{
    extern __shared__ double4 smem_raw[];
    EmisGemmSmem &sm = *reinterpret_cast<EmisGemmSmem *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int gid = lane >> 2, tig = lane & 3;
    const int ntile_n = wpitch / kEN;
    const int n0 = (int)(blockIdx.x % ntile_n) * kEN;
    const long long m0 = (long long)(blockIdx.x / ntile_n) * kEM;

    auto load_tile = [&](int buf, int k0) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int q = tid + 256 * c;   // row q / 8, 16-byte chunk q % 8
            const int r = q >> 3, ch = q & 7;
            const long long m = m0 + r;
            const bool ok = m < nrows;
            cp16(&sm.A[buf][r][ch * 2], N + (size_t)(ok ? m : 0) * NB + k0 + ch * 2, ok);
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int q = tid + 256 * c;   // row q / 32, chunk q % 32
            const int r = q >> 5, ch = q & 31;
            cp16(&sm.B[buf][r][ch * 2], W + (size_t)(k0 + r) * wpitch + n0 + ch * 2, true);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

    load_tile(0, 0);
    int buf = 0;
#pragma unroll 1
    for (int k0 = 0; k0 < NB; k0 += kEK) {
        if (k0 + kEK < NB) {
            load_tile(buf ^ 1, k0 + kEK);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kEK; kk += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; i++) af[i] = sm.A[buf][wm + 8 * i + gid][kk + tig];
#pragma unroll
            for (int j = 0; j < 4; j++) bf[j] = sm.B[buf][kk + tig][wn + 8 * j + gid];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) mma_f64(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        __syncthreads();
        buf ^= 1;
    }
    // fragment (i, j): C[wm + 8i + gid][wn + 8j + 2 tig + {0, 1}]
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const long long m = m0 + wm + 8 * i + gid;
        if (m >= nrows) continue;
        const double s = scale ? scale[(size_t)m * scale_stride] : 1.0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int k = n0 + wn + 8 * j + 2 * tig;
            if (k < ncols) out[(size_t)m * ncols + k] = acc[i][j][0] * s;
            if (k + 1 < ncols) out[(size_t)m * ncols + k + 1] = acc[i][j][1] * s;
        }
    }
}

// W[j][k] = fic[k][j] dp[j] (IC) or E_k / 2 beta_p[j] kern[k][j] c_j with c
// the trapezoid weights of Q_one: c_0 = dp_1, c_j = dp_j + dp_{j+1},
// c_{nb-1} = dp_{nb-1} (hadronic).  Zero past nbins.
__global__ void fold_weights_kernel(int nbins, int wpitch, const double *kern, const double *dp,
                                    const double *beta_p, const double *E, double *W)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NB * wpitch) return;
    const int j = i / wpitch, k = i % wpitch;
    double w = 0.0;
    if (k < nbins) {
        const double f = kern[(size_t)k * NB + j];
        if (!beta_p) {
            w = f * dp[j];
        } else {
            const double c = (j == 0) ? dp[1] : (j == NB - 1 ? dp[NB - 1] : dp[j] + dp[j + 1]);
            w = 0.5 * E[k] * (beta_p[j] * f * c);
        }
    }
    W[i] = w;
}

// The synchrotron emission with the table rows shared: tracers are sorted by
// their lower log-B plane ib (synch_plane_kernel + a radix sort), and a block
// of kSynWarps warps takes kSynWarps consecutive sorted tracers, one per
// warp.  For each frequency the block stages the rows K and log K of the
// planes its tracers interpolate between -- two or three planes when their
// ib values span at most two, which the sort makes the common case -- in
// shared memory, so each row is read once per block instead of once per
// tracer.  A block whose tracers span more planes reads the table directly.
// Per tracer: K = exp((1 - t) log K_ib + t log K_ib+1) where both ends are
// positive, the linear blend otherwise, clamped ends at t = 0 and 1.
constexpr int kSynWarps = 8;

__device__ __forceinline__ void synch_plane(double bval_in, double logb_min, double inv_dlogb, int nlogb, int &ib,
                                            double &tw)
{
    double bval = bval_in;
    if (!(bval > 0.0) || !isfinite(bval)) bval = 1.0e-30;
    const double lb = log10(bval / 1.0e-6);
    const double u = (lb - logb_min) * inv_dlogb;
    ib = (int)floor(u);
    if (ib < 0) ib = 0;
    if (ib > nlogb - 2) ib = nlogb - 2;
    tw = u - (double)ib;
    if (tw < 0.0) tw = 0.0;
    if (tw > 1.0) tw = 1.0;
}

__global__ void synch_plane_kernel(int ntracer, int nlogb, double logb_min, double inv_dlogb, const double *bfield,
                                   int *key, int *idx)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntracer) return;
    int ib;
    double tw;
    synch_plane(bfield[t], logb_min, inv_dlogb, nlogb, ib, tw);
    key[t] = ib;
    idx[t] = t;
}

struct SynRows {
    double K[3][NB], L[3][NB];
};

__global__ void __launch_bounds__(kSynWarps * 32, 3) synch_sorted_kernel(
    int ntracer, int nfreq, int nlogb, double logb_min, double inv_dlogb, SynchPrefactor sp, const double *K,
    const double *logK, const int *order, const double *bfield, const double *cre, const double *dp, double *out)
{
    constexpr int R = NB / 32;
    extern __shared__ double4 syn_smem[];
    SynRows &rows = *reinterpret_cast<SynRows *>(syn_smem);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long first = (long long)blockIdx.x * kSynWarps;
    const long long last = min((long long)ntracer, first + kSynWarps) - 1;
    const long long pos = first + w;
    const bool active = pos < ntracer;
    // the block's plane range (sorted: first and last tracer bound it)
    int ib_lo, ib_hi;
    double tw_unused;
    synch_plane(bfield[order[first]], logb_min, inv_dlogb, nlogb, ib_lo, tw_unused);
    synch_plane(bfield[order[last]], logb_min, inv_dlogb, nlogb, ib_hi, tw_unused);
    const bool staged = ib_hi - ib_lo <= 1;
    const int nplanes = staged ? ib_hi - ib_lo + 2 : 0;
    const int t = active ? order[pos] : 0;
    const double *N = cre + (size_t)t * NB;
    int stop = NB - 1;
    for (int j0 = 2; j0 < NB - 1; j0 += 32) {
        const int je = j0 + lane;
        const unsigned hit = __ballot_sync(kFull, je < NB - 1 && !(N[je + 1] > 0.0));
        if (hit) {
            stop = j0 + __ffs(hit) - 1;
            break;
        }
    }
    double nd[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int je = 32 * r + lane;
        nd[r] = (active && je >= 2 && je < stop) ? N[je] * dp[je] : 0.0;
    }
    int ib;
    double tw;
    synch_plane(active ? bfield[t] : 1.0, logb_min, inv_dlogb, nlogb, ib, tw);
    const double A = active ? sp.a0 * bfield[t] / sp.den1 / sp.den2 : 0.0;
    const int s0 = ib - ib_lo;   // staged row of plane ib
    for (int nf = 0; nf < nfreq; nf++) {
        if (staged) {
            __syncthreads();
            for (int i = threadIdx.x; i < nplanes * NB; i += blockDim.x) {
                const int pl = i / NB, je = i % NB;
                const size_t o = ((size_t)(ib_lo + pl) * nfreq + nf) * NB + je;
                rows.K[pl][je] = __ldg(K + o);
                rows.L[pl][je] = __ldg(logK + o);
            }
            __syncthreads();
        }
        if (!active) continue;
        const size_t o0 = ((size_t)ib * nfreq + nf) * NB, o1 = ((size_t)(ib + 1) * nfreq + nf) * NB;
        double sum = 0.0;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int je = 32 * r + lane;
            if (nd[r] == 0.0) continue;
            double Kv;
            if (tw <= 0.0) {
                Kv = staged ? rows.K[s0][je] : __ldg(K + o0 + je);
            } else if (tw >= 1.0) {
                Kv = staged ? rows.K[s0 + 1][je] : __ldg(K + o1 + je);
            } else {
                const double la = staged ? rows.L[s0][je] : __ldg(logK + o0 + je);
                const double lb = staged ? rows.L[s0 + 1][je] : __ldg(logK + o1 + je);
                if (!isnan(la) && !isnan(lb)) {
                    Kv = exp((1.0 - tw) * la + tw * lb);
                } else {
                    const double ka = staged ? rows.K[s0][je] : __ldg(K + o0 + je);
                    const double kb = staged ? rows.K[s0 + 1][je] : __ldg(K + o1 + je);
                    Kv = (1.0 - tw) * ka + tw * kb;
                }
            }
            sum += nd[r] * Kv;
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(kFull, sum, off);
        if (lane == 0) out[(size_t)t * nfreq + nf] = A * sum;
    }
}

// ---------------------------------------------------------------------------
// Host helpers.

// Band centres as the reference accumulates them: a = lo - d, then a += d and
// 10^a per band (fp_shared_core.c:1735-1742, tracer_fp_synch.c:103-109).
std::vector<double> log_grid(int n, double lo, double hi)
{
    std::vector<double> v(n);
    const double d = (hi - lo) / (double)n;
    double a = lo - d;
    for (int i = 0; i < n; i++) {
        a += d;
        v[i] = pow(10.0, a);
    }
    return v;
}

IcConsts ic_consts()
{
    // the CMB photon density prefactors of FP_Coef.c:391-413 (as tables.cu
    // builds them for the IC-cooling rows)
    const double meg = 9.11e-28;
    IcConsts k;
    k.cmb_pref = 8.0 * kPi * kC * kC * kC * pow(meg / kHPlanck, 3.0);
    k.cmb_pref_d = 8.0 * kPi * kC * kC * kC * pow(meg / 6.63e-27, 3.0);
    k.k_d = 1.38 * pow(10.0, -16.0);
    k.log10_90 = 90.0 * log(10.0);
    return k;
}

int fail_msg(int code, const char *msg)
{
    set_error(msg);
    return code;
}

// One-shot device blocks of the stateless entry points.
struct Blocks {
    std::vector<void *> ptrs;
    ~Blocks()
    {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t get(T **out, size_t n)
    {
        void *p = nullptr;
        const cudaError_t e = cudaMalloc(&p, n ? n * sizeof(T) : 8);
        if (e == cudaSuccess) ptrs.push_back(p);
        *out = static_cast<T *>(p);
        return e;
    }
};

enum TableKind { kTabGamma = 0, kTabNeutrino = 1, kTabIc = 2 };

// One kernel table [nbins][NB] into the device array d_out on stream st.
cudaError_t launch_table(int kind, int nbins, const double *d_E, const double *d_p, double z, double *d_out,
                         cudaStream_t st)
{
    const int n = nbins * NB;
    const int blocks = (n + 127) / 128;
    if (kind == kTabGamma) gamma_table_kernel<<<blocks, 128, 0, st>>>(nbins, d_E, d_p, d_out);
    else if (kind == kTabNeutrino) neutrino_table_kernel<<<blocks, 128, 0, st>>>(nbins, d_E, d_p, d_out);
    else ic_table_kernel<<<blocks, 128, 0, st>>>(ic_consts(), nbins, d_E, d_p, z, d_out);
    return cudaGetLastError();
}

// prepare_{gamma,neutrino,ic}_kernel_flat on the device: host grid in, host table out.
int table_host(int kind, const double *p_host, int nbins, double lo, double hi, double z, double *out)
{
    if (!p_host || !out || nbins <= 0) return fail_msg(-1, "invalid kernel-table arguments");
    const std::vector<double> E = log_grid(nbins, lo, hi);
    Blocks b;
    double *d_E, *d_p, *d_out;
    CROMA_CUDA(b.get(&d_E, nbins));
    CROMA_CUDA(b.get(&d_p, NB));
    CROMA_CUDA(b.get(&d_out, (size_t)nbins * NB));
    CROMA_CUDA(cudaMemcpy(d_E, E.data(), nbins * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_p, p_host, NB * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(launch_table(kind, nbins, d_E, d_p, z, d_out, 0));
    CROMA_CUDA(cudaMemcpy(out, d_out, (size_t)nbins * NB * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

// The synchrotron tables of tracer_fp_synch_data_init_tables
// (src/tracer_fp_synch.c:87-121) on the device: logx grid, log F, F, pitch
// angles and weights, frequencies, logy.
struct SynchBuild {
    int nx = 2750;
    double xmin = -25.0, xmax = 2.5;
    std::vector<double> logx, theta, w, nus;
    double *d_logx = nullptr, *d_logfx = nullptr, *d_logy = nullptr, *d_w = nullptr;
};

}  // namespace

// ---------------------------------------------------------------------------
// Resident emission of a context.
struct EmissionState {
    CromaB200EmissionSetup cfg{};
    int wp_ic = 0, wp_gamma = 0, wp_nu = 0;   // weight pitches (multiples of 64)
    double *d_block = nullptr;                // one device block for everything below
    double *d_K = nullptr, *d_logK = nullptr; // synchrotron [nlogb][nfreq][NB]
    double *d_w_ic = nullptr, *d_w_gamma = nullptr, *d_w_nu = nullptr;   // [NB][wp]
    double *d_fic = nullptr;                  // IC kernel [nbins_ic][NB] of ic_z
    double *d_nu_ic = nullptr, *d_p_e = nullptr;
    double ic_z = 0.0;
    int ic_valid = 0;
    int ic_rebuilt = 0;                       // the last run rebuilt the IC table (2 more launches)
    double inv_dlogb = 0.0;
    size_t bytes = 0;
    // device outputs of croma_b200_step_host (grow-only)
    double *d_out = nullptr;
    size_t out_bytes = 0;
    // tracer order of the synchrotron kernel (sorted by log-B plane)
    int *d_key = nullptr, *d_key_alt = nullptr, *d_idx = nullptr, *d_idx_alt = nullptr;
    void *d_sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    int sort_cap = 0;
};

void free_emission(Context &c)
{
    if (!c.emission) return;
    EmissionState *e = c.emission;
    if (e->d_block) dev_free(c, e->d_block);
    for (void *p : {(void *)e->d_key, (void *)e->d_key_alt, (void *)e->d_idx, (void *)e->d_idx_alt, e->d_sort_tmp,
                    (void *)e->d_out})
        if (p) dev_free(c, p);
    delete e;
    c.emission = nullptr;
}

namespace {

int pad64(int n) { return (n + 63) / 64 * 64; }

cudaError_t launch_gemm(int nrows, int ncols, int wpitch, const double *N, const double *W, const double *scale,
                        int scale_stride, double *out, cudaStream_t st)
{
    constexpr size_t smem = sizeof(EmisGemmSmem);
    static const cudaError_t attr =
        cudaFuncSetAttribute(emission_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr != cudaSuccess) return attr;
    const long long blocks = ((long long)nrows + kEM - 1) / kEM * (wpitch / kEN);
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    emission_gemm_kernel<<<(unsigned)blocks, 256, smem, st>>>(nrows, ncols, wpitch, N, W, scale, scale_stride, out);
    return cudaGetLastError();
}

int setup_emission(Context &c, const CromaB200EmissionSetup *s)
{
    if (!s) return fail_msg(-1, "null emission setup");
    if (s->nfreq < 0 || s->nbins_ic < 0 || s->nbins_gamma < 0 || s->nbins_nu < 0)
        return fail_msg(-1, "negative band count");
    if (s->nfreq > 0 && (s->ntheta_pitch <= 0 || s->nlogb < 2 || s->nlogb > 65536 || !(s->logb_max > s->logb_min)))
        return fail_msg(-1, "synchrotron needs ntheta_pitch > 0, 2 <= nlogb <= 65536 and logb_max > logb_min");
    if ((s->nfreq > 0 || s->nbins_ic > 0) && !(c.mp.species_mask & CROMA_SPECIES_ELECTRON))
        return fail_msg(-1, "synchrotron / IC emission needs the electron species");
    if ((s->nbins_gamma > 0 || s->nbins_nu > 0) && !(c.mp.species_mask & CROMA_SPECIES_PROTON))
        return fail_msg(-1, "gamma / neutrino emission needs the proton species");
    CROMA_CUDA(cudaSetDevice(c.device));
    free_emission(c);
    EmissionState *e = new EmissionState();
    c.emission = e;
    e->cfg = *s;
    e->wp_ic = pad64(s->nbins_ic);
    e->wp_gamma = pad64(s->nbins_gamma);
    e->wp_nu = pad64(s->nbins_nu);
    const size_t nsyn = (size_t)s->nlogb * s->nfreq * NB;
    const size_t total = (s->nfreq > 0 ? 2 * nsyn : 0) + (size_t)NB * (e->wp_ic + e->wp_gamma + e->wp_nu) +
                         (size_t)s->nbins_ic * NB + s->nbins_ic + NB;
    e->bytes = total * sizeof(double);
    CROMA_CUDA(dev_alloc(c, &e->d_block, e->bytes));
    double *p = e->d_block;
    if (s->nfreq > 0) {
        e->d_K = p; p += nsyn;
        e->d_logK = p; p += nsyn;
    }
    e->d_w_ic = p; p += (size_t)NB * e->wp_ic;
    e->d_w_gamma = p; p += (size_t)NB * e->wp_gamma;
    e->d_w_nu = p; p += (size_t)NB * e->wp_nu;
    e->d_fic = p; p += (size_t)s->nbins_ic * NB;
    e->d_nu_ic = p; p += s->nbins_ic;
    e->d_p_e = p; p += NB;
    cudaStream_t st = c.stream;
    CROMA_CUDA(cudaMemcpyAsync(e->d_p_e, c.h_p[1].data(), NB * sizeof(double), cudaMemcpyHostToDevice, st));
    // scratch of the build: released at the end (stream-ordered)
    std::vector<void *> scratch;
    struct Release {
        Context &c;
        std::vector<void *> &v;
        ~Release()
        {
            for (void *q : v) dev_free(c, q);
        }
    } rel{c, scratch};
    auto tmp = [&](double **out, size_t n) -> cudaError_t {
        const cudaError_t er = dev_alloc(c, out, n * sizeof(double));
        if (er == cudaSuccess) scratch.push_back(*out);
        return er;
    };
    // ---- hadronic weights (proton grid): kernel table, then the folded weights
    const std::vector<double> beta = [&] {
        std::vector<double> b(NB);
        for (int j = 0; j < NB; j++) {
            const double pj = c.h_p[0][j];
            b[j] = pj / sqrt(1.0 + pj * pj);
        }
        return b;
    }();
    for (int kind = kTabGamma; kind <= kTabNeutrino; kind++) {
        const int nb = kind == kTabGamma ? s->nbins_gamma : s->nbins_nu;
        if (nb <= 0) continue;
        const double lo = kind == kTabGamma ? s->egamma_min : s->enu_min;
        const double hi = kind == kTabGamma ? s->egamma_max : s->enu_max;
        const std::vector<double> E = log_grid(nb, lo, hi);
        double *d_E, *d_p, *d_beta, *d_dp, *d_kern;
        CROMA_CUDA(tmp(&d_E, nb));
        CROMA_CUDA(tmp(&d_p, NB));
        CROMA_CUDA(tmp(&d_beta, NB));
        CROMA_CUDA(tmp(&d_dp, NB));
        CROMA_CUDA(tmp(&d_kern, (size_t)nb * NB));
        CROMA_CUDA(cudaMemcpyAsync(d_E, E.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
        CROMA_CUDA(cudaMemcpyAsync(d_p, c.h_p[0].data(), NB * sizeof(double), cudaMemcpyHostToDevice, st));
        CROMA_CUDA(cudaMemcpyAsync(d_beta, beta.data(), NB * sizeof(double), cudaMemcpyHostToDevice, st));
        CROMA_CUDA(cudaMemcpyAsync(d_dp, c.h_dp[0].data(), NB * sizeof(double), cudaMemcpyHostToDevice, st));
        CROMA_CUDA(launch_table(kind, nb, d_E, d_p, 0.0, d_kern, st));
        const int wp = kind == kTabGamma ? e->wp_gamma : e->wp_nu;
        double *W = kind == kTabGamma ? e->d_w_gamma : e->d_w_nu;
        fold_weights_kernel<<<(NB * wp + 127) / 128, 128, 0, st>>>(nb, wp, d_kern, d_dp, d_beta, d_E, W);
        CROMA_CUDA(cudaGetLastError());
        // the host copies must outlive the asynchronous uploads
        CROMA_CUDA(cudaStreamSynchronize(st));
    }
    if (s->nbins_ic > 0) {
        const std::vector<double> nu = log_grid(s->nbins_ic, s->nu_min_ic, s->nu_max_ic);
        CROMA_CUDA(cudaMemcpyAsync(e->d_nu_ic, nu.data(), nu.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        CROMA_CUDA(cudaStreamSynchronize(st));
    }
    // ---- synchrotron: F(x), logy, pitch-kernel table, log K
    if (s->nfreq > 0) {
        SynchBuild b;
        const double dx = (b.xmax - b.xmin) / (double)b.nx;
        b.logx.resize(b.nx);
        for (int i = 0; i < b.nx; i++) b.logx[i] = b.xmin + dx * (double)i;
        const int nth = s->ntheta_pitch;
        b.theta.resize(nth);
        b.w.resize(nth);
        for (int k = 0; k < nth; k++) {
            b.theta[k] = (k + 0.5) * kPi / (double)nth;
            const double dth = kPi / (double)nth;
            b.w[k] = sin(b.theta[k]) * sin(b.theta[k]) * dth;
        }
        b.nus = log_grid(s->nfreq, s->nu_min_s, s->nu_max_s);
        double *d_theta, *d_nus, *d_p, *d_logy;
        CROMA_CUDA(tmp(&b.d_logx, b.nx));
        CROMA_CUDA(tmp(&b.d_logfx, b.nx));
        CROMA_CUDA(tmp(&d_theta, nth));
        CROMA_CUDA(tmp(&b.d_w, nth));
        CROMA_CUDA(tmp(&d_nus, s->nfreq));
        CROMA_CUDA(tmp(&d_p, NB));
        CROMA_CUDA(tmp(&d_logy, (size_t)s->nfreq * NB * nth));
        CROMA_CUDA(cudaMemcpyAsync(b.d_logx, b.logx.data(), b.nx * sizeof(double), cudaMemcpyHostToDevice, st));
        CROMA_CUDA(cudaMemcpyAsync(d_theta, b.theta.data(), nth * sizeof(double), cudaMemcpyHostToDevice, st));
        CROMA_CUDA(cudaMemcpyAsync(b.d_w, b.w.data(), nth * sizeof(double), cudaMemcpyHostToDevice, st));
        CROMA_CUDA(cudaMemcpyAsync(d_nus, b.nus.data(), s->nfreq * sizeof(double), cudaMemcpyHostToDevice, st));
        CROMA_CUDA(cudaMemcpyAsync(d_p, c.h_p[1].data(), NB * sizeof(double), cudaMemcpyHostToDevice, st));
        synch_logfx_kernel<<<(b.nx + 7) / 8, 256, 0, st>>>(b.nx, b.d_logx, b.d_logfx);
        CROMA_CUDA(cudaGetLastError());
        int dev = 0, nsm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        synch_logy_kernel<<<8 * nsm, 256, 0, st>>>(s->nfreq, nth, d_nus, d_p, d_theta, d_logy);
        CROMA_CUDA(cudaGetLastError());
        // the last table value F(x_last) = 10^logF (fx_tab, tracer_fp_synch.c:97)
        double logf_last = 0.0;
        CROMA_CUDA(cudaMemcpyAsync(&logf_last, b.d_logfx + (b.nx - 1), sizeof(double), cudaMemcpyDeviceToHost, st));
        CROMA_CUDA(cudaStreamSynchronize(st));
        SynchFx F{};
        F.nx = b.nx;
        F.xmin = b.xmin;
        F.inv_dlogx = 1.0 / (b.logx[1] - b.logx[0]);
        F.logx_last = b.logx[b.nx - 1];
        F.fx_last = pow(10.0, logf_last);
        F.logx_tab = b.d_logx;
        F.logfx_tab = b.d_logfx;
        e->inv_dlogb = (double)(s->nlogb - 1) / (s->logb_max - s->logb_min);
        synch_pitch_table_kernel<<<16 * nsm, 256, 0, st>>>(F, s->nfreq, nth, s->nlogb, s->logb_min, e->inv_dlogb,
                                                           d_logy, b.d_w, e->d_K);
        CROMA_CUDA(cudaGetLastError());
        log_table_kernel<<<8 * nsm, 256, 0, st>>>((long long)nsyn, e->d_K, e->d_logK);
        CROMA_CUDA(cudaGetLastError());
        CROMA_CUDA(cudaStreamSynchronize(st));
    }
    e->ic_valid = 0;
    return 0;
}

}  // namespace

int emission_run(Context &c, const double *bg, double z, double *eps_syn, double *eps_ic, double *eps_gamma,
                 double *eps_nu)
{
    EmissionState *e = c.emission;
    if (!e) return fail_msg(-1, "emission not set up: call croma_b200_emission_setup first");
    if (c.ntracer <= 0 || !c.d_cre || !c.d_crp) return fail_msg(-1, "no resident spectra");
    const CromaB200EmissionSetup &s = e->cfg;
    const int n = c.ntracer;
    cudaStream_t st = c.stream;
    e->ic_rebuilt = 0;
    if (eps_ic && s.nbins_ic > 0) {
        if (!e->ic_valid || e->ic_z != z) {
            e->ic_rebuilt = 1;
            CROMA_CUDA(launch_table(kTabIc, s.nbins_ic, e->d_nu_ic, e->d_p_e, z, e->d_fic, st));
            fold_weights_kernel<<<(NB * e->wp_ic + 127) / 128, 128, 0, st>>>(s.nbins_ic, e->wp_ic, e->d_fic,
                                                                             c.gt.s[1].dp, nullptr, nullptr,
                                                                             e->d_w_ic);
            CROMA_CUDA(cudaGetLastError());
            e->ic_z = z;
            e->ic_valid = 1;
        }
        CROMA_CUDA(launch_gemm(n, s.nbins_ic, e->wp_ic, c.d_cre, e->d_w_ic, nullptr, 0, eps_ic, st));
    }
    // n_gas is field 0 of the field-major background [8][ntracer]
    if (eps_gamma && s.nbins_gamma > 0)
        CROMA_CUDA(launch_gemm(n, s.nbins_gamma, e->wp_gamma, c.d_crp, e->d_w_gamma, bg, 1, eps_gamma, st));
    if (eps_nu && s.nbins_nu > 0)
        CROMA_CUDA(launch_gemm(n, s.nbins_nu, e->wp_nu, c.d_crp, e->d_w_nu, bg, 1, eps_nu, st));
    if (eps_syn && s.nfreq > 0) {
        const double *bfield = bg + 2 * (size_t)n;
        if (e->sort_cap < n) {
            for (void *p : {(void *)e->d_key, (void *)e->d_key_alt, (void *)e->d_idx, (void *)e->d_idx_alt,
                            e->d_sort_tmp})
                if (p) dev_free(c, p);
            e->d_key = e->d_key_alt = e->d_idx = e->d_idx_alt = nullptr;
            e->d_sort_tmp = nullptr;
            e->sort_cap = 0;
            CROMA_CUDA(dev_alloc(c, &e->d_key, (size_t)n * sizeof(int)));
            CROMA_CUDA(dev_alloc(c, &e->d_key_alt, (size_t)n * sizeof(int)));
            CROMA_CUDA(dev_alloc(c, &e->d_idx, (size_t)n * sizeof(int)));
            CROMA_CUDA(dev_alloc(c, &e->d_idx_alt, (size_t)n * sizeof(int)));
            cub::DoubleBuffer<int> kb(e->d_key, e->d_key_alt), vb(e->d_idx, e->d_idx_alt);
            size_t bytes = 0;
            CROMA_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kb, vb, n, 0, 16, st));
            CROMA_CUDA(dev_alloc_bytes(c, &e->d_sort_tmp, bytes ? bytes : 16));
            e->sort_tmp_bytes = bytes;
            e->sort_cap = n;
        }
        synch_plane_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, s.nlogb, s.logb_min, e->inv_dlogb, bfield, e->d_key,
                                                             e->d_idx);
        CROMA_CUDA(cudaGetLastError());
        // plane indices are below 2^16 (nlogb is bounded by the table's size)
        cub::DoubleBuffer<int> kb(e->d_key, e->d_key_alt), vb(e->d_idx, e->d_idx_alt);
        size_t bytes = e->sort_tmp_bytes;
        CROMA_CUDA(cub::DeviceRadixSort::SortPairs(e->d_sort_tmp, bytes, kb, vb, n, 0, 16, st));
        constexpr size_t smem = sizeof(SynRows);
        static const cudaError_t attr =
            cudaFuncSetAttribute(synch_sorted_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        CROMA_CUDA(attr);
        synch_sorted_kernel<<<(n + kSynWarps - 1) / kSynWarps, kSynWarps * 32, smem, st>>>(
            n, s.nfreq, s.nlogb, s.logb_min, e->inv_dlogb, synch_prefactor(), e->d_K, e->d_logK, vb.Current(),
            bfield, c.d_cre, c.gt.s[1].dp, eps_syn);
        CROMA_CUDA(cudaGetLastError());
    }
    return 0;
}

int emission_setup(Context &c, const CromaB200EmissionSetup *s) { return setup_emission(c, s); }

const CromaB200EmissionSetup &emission_config(const Context &c) { return c.emission->cfg; }

cudaError_t emission_out_block(Context &c, size_t bytes, double **out)
{
    EmissionState *e = c.emission;
    if (!e) return cudaErrorInvalidValue;
    if (e->out_bytes < bytes) {
        if (e->d_out) dev_free(c, e->d_out);
        e->d_out = nullptr;
        e->out_bytes = 0;
        const cudaError_t er = dev_alloc(c, &e->d_out, bytes);
        if (er != cudaSuccess) return er;
        e->out_bytes = bytes;
    }
    *out = e->d_out;
    return cudaSuccess;
}

int emission_launches(const Context &c, bool syn, bool ic, bool gamma, bool nu)
{
    const EmissionState *e = c.emission;
    if (!e) return 0;
    return 3 * (syn && e->cfg.nfreq > 0) + (ic && e->cfg.nbins_ic > 0) * (1 + 2 * e->ic_rebuilt) +
           (gamma && e->cfg.nbins_gamma > 0) + (nu && e->cfg.nbins_nu > 0);
}

int emission_tables(Context &c, int which, double *out)
{
    EmissionState *e = c.emission;
    if (!e || !out) return fail_msg(-1, "emission not set up or null output");
    const CromaB200EmissionSetup &s = e->cfg;
    const double *src = nullptr;
    size_t n = 0;
    if (which == CROMA_EMIS_TABLE_SYNCH && s.nfreq > 0) {
        src = e->d_K;
        n = (size_t)s.nlogb * s.nfreq * NB;
    } else if (which == CROMA_EMIS_TABLE_IC && s.nbins_ic > 0 && e->ic_valid) {
        src = e->d_fic;
        n = (size_t)s.nbins_ic * NB;
    }
    if (!src) return fail_msg(-1, "table not available (kind not set up, or IC not built yet)");
    CROMA_CUDA(cudaMemcpyAsync(out, src, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    return 0;
}

}  // namespace croma

using namespace croma;

extern "C" {

int synch_logfx_table_cuda(int nx, const double *logx, double *logfx_out)
{
    if (nx <= 0 || !logx || !logfx_out) return fail_msg(-1, "invalid F(x) table arguments");
    Blocks b;
    double *d_x, *d_f;
    CROMA_CUDA(b.get(&d_x, nx));
    CROMA_CUDA(b.get(&d_f, nx));
    CROMA_CUDA(cudaMemcpy(d_x, logx, nx * sizeof(double), cudaMemcpyHostToDevice));
    synch_logfx_kernel<<<(nx + 7) / 8, 256>>>(nx, d_x, d_f);
    CROMA_CUDA(cudaGetLastError());
    CROMA_CUDA(cudaMemcpy(logfx_out, d_f, nx * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int prepare_gamma_kernel_flat_cuda(const CRspectrum *crp, int nbins, double egamma_min, double egamma_max,
                                   double *fga_flat)
{
    if (!crp) return fail_msg(-1, "null proton grid");
    return table_host(kTabGamma, crp->p, nbins, egamma_min, egamma_max, 0.0, fga_flat);
}

int prepare_neutrino_kernel_flat_cuda(const CRspectrum *crp, int nbins, double enu_min, double enu_max,
                                      double *fnu_flat)
{
    if (!crp) return fail_msg(-1, "null proton grid");
    return table_host(kTabNeutrino, crp->p, nbins, enu_min, enu_max, 0.0, fnu_flat);
}

int prepare_ic_kernel_flat_cuda(const CRspectrum *cre, int nbins, double nu_min, double nu_max, double z,
                                double *fic_flat)
{
    if (!cre) return fail_msg(-1, "null electron grid");
    return table_host(kTabIc, cre->p, nbins, nu_min, nu_max, z, fic_flat);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Native C ABI (include/croma_b200.h).
struct CromaB200Context {
    croma::Context impl;
};

extern "C" {

int croma_b200_emission_setup(CromaB200Context *ctx, const CromaB200EmissionSetup *setup)
{
    if (!ctx) return fail_msg(-1, "null context");
    return emission_setup(ctx->impl, setup);
}

int croma_b200_emission_run(CromaB200Context *ctx, const double *bg, double z, double *eps_syn, double *eps_ic,
                            double *eps_gamma, double *eps_nu, int on_device)
{
    if (!ctx || !bg) return fail_msg(-1, "null context or background");
    Context &c = ctx->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    if (!c.emission) return fail_msg(-1, "emission not set up: call croma_b200_emission_setup first");
    if (on_device) return emission_run(c, bg, z, eps_syn, eps_ic, eps_gamma, eps_nu);
    // host background and outputs: fields 0..2 up, the outputs back
    const CromaB200EmissionSetup &s = c.emission->cfg;
    const size_t n = (size_t)(c.ntracer > 0 ? c.ntracer : 0);
    if (n == 0) return fail_msg(-1, "no resident spectra");
    const int cols[4] = {eps_syn ? s.nfreq : 0, eps_ic ? s.nbins_ic : 0, eps_gamma ? s.nbins_gamma : 0,
                         eps_nu ? s.nbins_nu : 0};
    double *host_out[4] = {eps_syn, eps_ic, eps_gamma, eps_nu};
    size_t total = 3 * n;
    for (int k = 0; k < 4; k++) total += n * (size_t)cols[k];
    double *blk = nullptr;
    CROMA_CUDA(dev_alloc(c, &blk, total * sizeof(double)));
    struct Free {
        Context &c;
        double *p;
        ~Free() { dev_free(c, p); }
    } guard{c, blk};
    CROMA_CUDA(cudaMemcpyAsync(blk, bg, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    double *dev_out[4];
    double *p = blk + 3 * n;
    for (int k = 0; k < 4; k++) {
        dev_out[k] = cols[k] ? p : nullptr;
        p += n * (size_t)cols[k];
    }
    const int rc = emission_run(c, blk, z, dev_out[0], dev_out[1], dev_out[2], dev_out[3]);
    if (rc) return rc;
    for (int k = 0; k < 4; k++)
        if (cols[k])
            CROMA_CUDA(cudaMemcpyAsync(host_out[k], dev_out[k], n * cols[k] * sizeof(double), cudaMemcpyDeviceToHost,
                                       c.stream));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    return 0;
}

int croma_b200_emission_table(CromaB200Context *ctx, int which, double *out)
{
    if (!ctx) return fail_msg(-1, "null context");
    CROMA_CUDA(cudaSetDevice(ctx->impl.device));
    return emission_tables(ctx->impl, which, out);
}

}  // extern "C"
