// background.cu -- the per-tracer background of a snapshot on the device.
//
// The reference prepares it on the host, per tracer, from the raw fields of
// a tracer snapshot: tracer_load_hdf5_raw_snapshot_slice scales the density
// by dUnit and the field by sqrt(4 pi dUnit) vUnit
// (src/tracer_fp_background.c:1189-1197, :955-957), and
// tracer_prepare_background_from_raw (:1206-1263) calls
// prepare_background_cell (src/fp_shared_core.c:866-932) with div v in
// Gyr^-1, curl v in s^-1, the target turbulence scale L_turb_target_kpc and
// the temperature-floor and curl-interpolation switches of the run loop
// (src/tracer_fp.c:917-1015).  Here one thread per tracer does the same
// arithmetic and writes the eight fields the update reads, field-major
// [8][ntracer] in the order of tracer_store_background_history_slot
// (:324-342): n_gas, kT (GeV), B_eff, div v (Gyr^-1), L_turb (Mpc),
// dv_imc, c_s, beta_pl.  The helper physics: c_sound (src/FP_Coef.c:916),
// dv_limit (:622), B_dynamo (:929).
#include <algorithm>
#include <cmath>

#include "croma_ctx.cuh"

namespace croma {
namespace {

constexpr double kBgKB = 8.62e-5;         // eV / K (src/CONSTANTS.c:12)
constexpr double kBgC = 2.999e10;         // cm / s
constexpr double kBgEV = 1.6e-12;         // erg
constexpr double kBgMpc = 3.0857e24;      // cm
constexpr double kBgKpc = 3.0857e21;      // cm (src/tracer_fp_background.c:37)
constexpr double kBgGyr = 3.1536e16;      // s  (src/tracer_fp_background.c:36)

struct BgArgs {
    CromaB200RawSnapshot r;
    CromaB200BackgroundParams p;
    int n;
    double *out;
    unsigned *err;
};

__global__ void __launch_bounds__(256) background_kernel(BgArgs a)
{
    const CromaB200RawSnapshot &r = a.r;
    const CromaB200BackgroundParams &p = a.p;
    const double target = p.l_turb_target_kpc * kBgKpc;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const double rho = r.density[i] * r.c_dens;
        const double bx = r.bx[i] * r.c_mag, by = r.by[i] * r.c_mag, bz = r.bz[i] * r.c_mag;
        if (!(rho > 0.0) || !(target > 0.0)) {   // prepare_background_cell returns -1
            atomicOr(a.err, 1u);
            for (int f = 0; f < 8; f++) a.out[(size_t)f * a.n + i] = 0.0;
            continue;
        }
        double temp = r.temp_K[i];
        if (r.apply_temp_floor && temp < 1.0e4) temp = 1.0e4;
        double curl = 1.0 * r.curl_v[i];
        if (r.allow_curl_interp && curl == 0.0 && r.z_next != r.z_prev) {
            const double cp = 1.0 * r.curl_v_prev[i], cn = 1.0 * r.curl_v_next[i];
            curl = __dadd_rn(__dmul_rn(__ddiv_rn(__dsub_rn(cn, cp), __dsub_rn(r.z_next, r.z_prev)),
                                       __dsub_rn(r.z_curr, r.z_prev)),
                             cp);
        }
        const double lraw = r.l_turb_cm ? r.l_turb_cm[i] : 0.0;
        const double lt = (lraw > 0.0) ? lraw : target;
        double dv = __dmul_rn(curl, lt);
        const double cs = __dmul_rn(sqrt(__ddiv_rn(__dmul_rn(__dmul_rn(5.0 / 3.0, kBgKB), temp),
                                                   __dmul_rn(__dmul_rn(p.mu_mol, 0.938), 1.0e9))),
                                    kBgC);
        dv = __dmul_rn(dv, pow(__ddiv_rn(target, lt), 0.3333));
        if (p.mach_limit > 0.0 && cs > 0.0 && __ddiv_rn(dv, cs) > p.mach_limit) dv = __dmul_rn(p.mach_limit, cs);
        const double b_sim = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(bx, bx), __dmul_rn(by, by)), __dmul_rn(bz, bz)));
        const double b_dyn =
            sqrt(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(4.0 * M_PI, p.eta_B), rho), dv), dv));
        const double b_eff = p.bfield_mode == 1 ? b_sim : (p.bfield_mode == 2 ? b_dyn : fmax(b_dyn, b_sim));
        const double n_gas = __ddiv_rn(rho, __dmul_rn(1.6e-24, p.mu_mol));
        const double beta = b_eff > 0.0
            ? __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(n_gas, kBgKB), temp), kBgEV),
                        __ddiv_rn(__dmul_rn(b_eff, b_eff), 8.0 * M_PI))
            : 1.0e10;
        const size_t N = (size_t)a.n;
        a.out[0 * N + i] = n_gas;
        a.out[1 * N + i] = __dmul_rn(__dmul_rn(kBgKB, temp), 1.0e-9);
        a.out[2 * N + i] = b_eff;
        a.out[3 * N + i] = __dmul_rn(__dmul_rn(1.0, r.div_v[i]), kBgGyr);
        a.out[4 * N + i] = __ddiv_rn(target, kBgMpc);
        a.out[5 * N + i] = dv;
        a.out[6 * N + i] = cs;
        a.out[7 * N + i] = beta;
    }
}

}  // namespace
}  // namespace croma

using namespace croma;

struct CromaB200Context {
    croma::Context impl;
};

extern "C" int croma_b200_background_prepare(CromaB200Context *ctx, int ntracer, const CromaB200RawSnapshot *raw,
                                             const CromaB200BackgroundParams *prm, int on_device, double *bg)
{
    if (!raw || !prm || !bg || ntracer < 0) { set_error("background_prepare: invalid arguments"); return -1; }
    if (ntracer == 0) return 0;
    const CromaB200RawSnapshot &r = *raw;
    if (!r.temp_K || !r.density || !r.bx || !r.by || !r.bz || !r.div_v || !r.curl_v) {
        set_error("background_prepare: a required raw field is null");
        return -1;
    }
    if (r.allow_curl_interp && (!r.curl_v_prev || !r.curl_v_next)) {
        set_error("background_prepare: curl interpolation needs curl_v_prev and curl_v_next");
        return -1;
    }
    if (prm->bfield_mode < 0 || prm->bfield_mode > 2) { set_error("background_prepare: bfield_mode must be 0, 1 or 2"); return -1; }
    cudaStream_t st = ctx ? ctx->impl.stream : nullptr;
    const size_t n = (size_t)ntracer;
    // host arrays go up into one device block: 10 raw fields, the output, the error word
    double *blk = nullptr, *d_host_out = nullptr;
    unsigned *d_err = nullptr;
    CromaB200RawSnapshot d = r;
    unsigned herr = 0;
    cudaError_t e = cudaSuccess;
    const char *what = "background_prepare";
    if (!on_device) {
        e = cudaMallocAsync(&blk, (10 * n) * sizeof(double) + 256, st);
        if (e == cudaSuccess) e = cudaMallocAsync(&d_host_out, 8 * n * sizeof(double), st);
        const double *src[10] = {r.temp_K, r.density, r.bx, r.by, r.bz, r.div_v, r.curl_v_prev, r.curl_v,
                                 r.curl_v_next, r.l_turb_cm};
        const double **dst[10] = {&d.temp_K, &d.density, &d.bx, &d.by, &d.bz, &d.div_v, &d.curl_v_prev, &d.curl_v,
                                  &d.curl_v_next, &d.l_turb_cm};
        for (int f = 0; f < 10 && e == cudaSuccess; f++) {
            if (!src[f]) { *dst[f] = nullptr; continue; }
            double *p = blk + (size_t)f * n;
            e = cudaMemcpyAsync(p, src[f], n * sizeof(double), cudaMemcpyHostToDevice, st);
            *dst[f] = p;
        }
        if (e == cudaSuccess) d_err = reinterpret_cast<unsigned *>(blk + 10 * n);
    } else {
        e = cudaMallocAsync(&d_err, 256, st);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) {
        BgArgs a{d, *prm, ntracer, on_device ? bg : d_host_out, d_err};
        const int blocks = (int)std::min<size_t>((n + 255) / 256, 65535);
        background_kernel<<<blocks, 256, 0, st>>>(a);
        e = cudaGetLastError();
        what = "background_kernel";
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && !on_device)
        e = cudaMemcpyAsync(bg, d_host_out, 8 * n * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    // released on every path
    if (d_host_out) cudaFreeAsync(d_host_out, st);
    if (blk) cudaFreeAsync(blk, st);
    if (on_device && d_err) cudaFreeAsync(d_err, st);
    if (e != cudaSuccess) return cuda_fail(e, what);
    if (herr) {
        set_error("background_prepare: a tracer has density <= 0 (or the target turbulence scale <= 0); "
                  "its fields are set to 0");
        return -2;
    }
    return 0;
}
