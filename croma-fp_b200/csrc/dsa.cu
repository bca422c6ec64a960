// dsa.cu -- per-snapshot DSA (diffusive shock acceleration) injection into the
// device-resident tracer spectra, one warp per tracer.
//
// For every tracer whose shock fields pass the reference's checks the warp
//   1. resolves the upstream state (Mach number, temperature, density,
//      speed; tracer_dsa_resolve_tracer_input, src/tracer_fp_dsa.c:26-108),
//   2. builds the fresh proton spectrum: efficiency eta(M) (the eight models
//      of src/DSA_MODELS.c:262-468), slope q = 3r/(r-1), injection momentum
//      chi p_th, and the normalisation from a 4000-interval Simpson integral of
//      the kinetic-energy density (src/DSA_MODELS.c:690-776) whose terms are
//      split over the lanes and combined by a shuffle tree,
//   3. builds the suprathermal electron spectrum normalised to the protons at
//      the proton injection momentum (src/DSA_MODELS.c:1022-1070),
//   4. optionally computes the reacceleration of the pre-shock spectra
//      (positive_delta / drury83 with its eta cap and the adiabatic part,
//      src/tracer_fp_dsa_reacc.c:60-236): the cumulative momentum integrals
//      run as warp scans over 32-bin chunks, the energy sums as shuffle trees,
//   5. adds source x V_downstream to the spectra (tracer_state mode) or
//      source x V_downstream / dt to the per-snapshot sources (tracer_source
//      mode), as tracer_fp_apply_dsa_tracer_injection_snapshot
//      (src/tracer_fp_dsa.c:184-565) does.
// The sums are reordered (lanes, scans) against the reference's sequential
// loops, so results agree with it to rounding.
#include "croma_segment.cuh"

namespace croma {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr double kMpG = 1.67262192369e-24;
constexpr double kMeG = 9.1093837015e-28;
constexpr double kKbCgs = 1.380649e-16;
constexpr double kCExact = 2.99792458e10;   // the DSA model code's speed of light
constexpr double kCCroma = 2.999e10;        // CROMA's c, used by the tracer energies
constexpr double k4Pi = 12.566370614359172;
constexpr double kMsunG = 1.99e33;
constexpr double kPiD = 3.14159265358979323846;
constexpr int kDsaWarps = 4;

struct DsaModelCoef {
    int family, reacc;
    double xcr0, b[5], mach_crit, scale;
};

// Efficiency model table, in DSAModelID order (src/DSA_MODELS.c:262-350).
__constant__ DsaModelCoef c_models[8] = {
    {0, 0, 0.0, {5.46, -9.78, 4.17, -0.33, 0.57}, 1.0, 1.0},
    {0, 1, 0.3, {0.24, -1.56, 2.8, 0.512, 0.557}, 1.0, 1.0},
    {1, 0, 0.0, {-2.87, 9.67, -8.88, 1.94, 0.18}, 2.0, 1.0},
    {1, 1, 0.05, {-0.72, 2.73, -3.29, 1.34, 0.19}, 2.0, 1.0},
    {1, 0, 0.0, {-2.87, 9.67, -8.88, 1.94, 0.18}, 2.0, 0.5},
    {1, 1, 0.05, {-0.72, 2.73, -3.29, 1.34, 0.19}, 2.0, 0.5},
    {2, 0, 0.0, {-1.5255, 2.4026, -1.2534, 0.2215, 0.0336}, 2.25, 1.0},
    {2, 1, 0.05, {0.3965, -0.21898, -0.2074, 0.1319, 0.0351}, 2.25, 1.0}};

struct DsaArgs {
    CromaB200DsaParams prm;
    // shock fields [ntracer] on the device (null = absent)
    const double *mach, *prestemp, *presden, *pre_density_cgs, *upstream_speed_cgs, *shock_side_code;
    const double *dsa_trigger, *dsa_mach, *dsa_pre_density, *dsa_flux;
    int has_dsa;
    int ntracer;
    double density_unit, dt_gyr;
    int mode, reacc;
    // spectra and sources: element (t, j) at base + t * ts + j * js
    double *crp, *cre, *qpi, *qepri;
    size_t ts, js;
    unsigned char *dis;
    const double *mass;           // [ntracer] solar masses
    const double *p[2], *dp[2];   // FP grids
    const double *dsa_p;          // [2][NB] DSA-grid momenta at the FP bins
    unsigned *count;
};

__device__ double quartic_over_m4(double m, const double *b)
{
    if (m <= 0.0) return 0.0;
    const double x = m - 1.0;
    return (b[0] + b[1] * x + b[2] * x * x + b[3] * x * x * x + b[4] * x * x * x * x) / (m * m * m * m);
}

__device__ double dsa_eta(double m, int id)
{
    if (id < 0 || id >= 8) return 0.0;
    const DsaModelCoef &md = c_models[id];
    if (m < md.mach_crit) return 0.0;
    const double poly = quartic_over_m4(m, md.b);
    double eta;
    if (md.family == 0 && !md.reacc) {
        eta = (m <= 2.0) ? 1.96e-3 * (m * m - 1.0) : poly;
    } else if (md.family == 0) {
        if (m <= 1.5) {
            const double g = 5.0 / 3.0, m2 = m * m;
            const double xs = (g + 1.0) / (g - 1.0 + 2.0 / m2);
            const double d0 = 2.0 * (((2.0 * g * m2 - g + 1.0) / (g + 1.0)) - pow(xs, g)) /
                              (g * (g - 1.0) * m2 * xs);
            eta = 1.025 * d0;
        } else {
            eta = poly;
        }
    } else if (md.family == 1 && !md.reacc) {
        if (m <= 5.0) eta = -0.0005950569221922047 + 1.880258286365841e-5 * pow(m, 5.334076006529829);
        else if (m <= 15.0) eta = poly;
        else eta = 0.21152;
    } else if (md.family == 1) {
        eta = (m <= 17.7) ? poly : 0.2055;
    } else {
        eta = (m <= 34.0) ? poly : 0.0348;
    }
    eta *= md.scale;
    return eta < 0.0 ? 0.0 : eta;
}

__device__ double compression_ratio(double m, double g)
{
    if (m <= 1.0 || g <= 1.0) return 1.0;
    const double m2 = m * m;
    const double den = (g - 1.0) * m2 + 2.0;
    if (den <= 0.0) return 1.0;
    return (g + 1.0) * m2 / den;
}

__device__ double injection_momentum(double temp, double chi, double mass_g)
{
    if (chi <= 0.0 || temp <= 0.0) return 0.0;
    const double th = 2.0 * kKbCgs * temp / (mass_g * kCExact * kCExact);
    if (th <= 0.0) return 0.0;
    return chi * sqrt(th);
}

__device__ double spectrum_shape(double p, double pinj, double q, double pmax)
{
    if (p <= 0.0 || pinj <= 0.0 || pmax <= 0.0 || p < pinj) return 0.0;
    const double rm = p / pmax;
    double e = -rm * rm;
    e = fmin(fmax(e, -700.0), 700.0);
    return pow(p / pinj, -q) * exp(e);
}

__device__ double energy_integrand(double p, double pinj, double q, double pmax)
{
    if (p <= 0.0 || p < pinj) return 0.0;
    return (sqrt(1.0 + p * p) - 1.0) * p * p * spectrum_shape(p, pinj, q, pmax);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
    return v;
}

// Inclusive prefix sum over the warp.
__device__ __forceinline__ double warp_scan(double v, int lane)
{
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double o = __shfl_up_sync(kFull, v, off);
        if (lane >= off) v += o;
    }
    return v;
}

// 4 pi m_p c^2 x Simpson integral of the energy integrand over [p_inj, p_max]
__device__ double proton_edens_unit(double pinj, double q, double pmax, int lane)
{
    if (pinj <= 0.0 || pmax <= 0.0 || pmax <= pinj) return 0.0;
    constexpr int nstep = 4000;
    const double h = (pmax - pinj) / (double)nstep;
    double s = 0.0;
    for (int i = 1 + lane; i < nstep; i += 32) {
        const double p = pinj + h * (double)i;
        s += ((i % 2) ? 4.0 : 2.0) * energy_integrand(p, pinj, q, pmax);
    }
    s = warp_sum(s);
    s += energy_integrand(pinj, pinj, q, pmax) + energy_integrand(pmax, pinj, q, pmax);
    return k4Pi * kMpG * kCExact * kCExact * (s * h / 3.0);
}

__device__ double source_dp(double A, double pinj, double q, double pmax, double p)
{
    if (p <= 0.0 || p < pinj || p > pmax) return 0.0;
    const double f = A * pow(p / pinj, -q) * exp(-(p / pmax) * (p / pmax));
    if (f <= 0.0) return 0.0;
    return k4Pi * p * p * f;
}

__device__ __forceinline__ double ekin_erg(double p, int electron)
{
    const double m = electron ? kMeG : kMpG;
    return m * kCCroma * kCCroma * (sqrt(1.0 + p * p) - 1.0);
}

__device__ bool resolve_input(const DsaArgs &A, int t, double &mach, double &temp, double &rho1,
                              double &u1)
{
    const CromaB200DsaParams &prm = A.prm;
    if (A.has_dsa) {
        if (!A.dsa_trigger || !A.dsa_mach || !A.dsa_pre_density || !A.dsa_flux) return false;
        if (!(A.dsa_trigger[t] > 0.5)) return false;
        const double flux = A.dsa_flux[t], m = A.dsa_mach[t];
        const double r = A.dsa_pre_density[t] * A.density_unit;
        if (!(m >= prm.min_mach) || !isfinite(m) || !(r > 0.0) || !isfinite(r)) return false;
        if (!(flux > 0.0) || !isfinite(flux)) return false;
        const double u = cbrt(2.0 * flux / r);
        if (!(u > 0.0) || !isfinite(u)) return false;
        const double T = (prm.mu_mol * kMpG / (prm.gamma_gas * kKbCgs)) * (u * u) / (m * m);
        if (!(T > 0.0) || !isfinite(T)) return false;
        mach = m; temp = T; rho1 = r; u1 = u;
        return true;
    }
    if (!A.mach || !A.prestemp || !A.presden) return false;
    const double m = A.mach[t], T = A.prestemp[t];
    if (!(m >= prm.min_mach) || !(T > 0.0) || !isfinite(m) || !isfinite(T)) return false;
    if (A.shock_side_code) {
        const int side = (int)floor(A.shock_side_code[t] + 0.5);
        if (side == -1 || side == 99) return false;
    }
    const double r = (A.pre_density_cgs && A.pre_density_cgs[t] > 0.0) ? A.pre_density_cgs[t]
                                                                       : A.presden[t] * A.density_unit;
    if (!(r > 0.0) || !isfinite(r)) return false;
    const double u = (A.upstream_speed_cgs && A.upstream_speed_cgs[t] > 0.0)
                   ? A.upstream_speed_cgs[t]
                   : m * sqrt(prm.gamma_gas * kKbCgs * T / (prm.mu_mol * kMpG));
    if (!(u > 0.0) || !isfinite(u)) return false;
    mach = m; temp = T; rho1 = r; u1 = u;
    return true;
}

// Per-warp shared rows: reacceleration deltas and adiabatic deltas of both
// species.
struct DsaSmem {
    double dlt[2][NB], ad[2][NB];
};

// positive_delta (tracer_fp_dsa_reacc.c:60-103): deltas and their energy density
__device__ double reacc_positive(const DsaArgs &A, int s, const double *N, double vdown, double q,
                                 double pmin, double *dlt, int lane)
{
    const double *p = A.p[s], *dp = A.dp[s];
    double carry = 0.0, de = 0.0;
    for (int j0 = 0; j0 < NB; j0 += 32) {
        const int j = j0 + lane;
        const bool use = j >= 1 && p[j] > 0.0 && p[j] >= pmin;
        const double cur = N[j * A.js] / vdown;
        double term = 0.0;
        if (use) term = pow(p[j], q - 1.0) * (cur / (4.0 * kPiD * p[j] * p[j])) * dp[j];
        const double incl = warp_scan(term, lane);
        const double integral = carry + incl;
        carry += __shfl_sync(kFull, incl, 31);
        double d = 0.0;
        if (use) {
            const double re = 4.0 * kPiD * p[j] * p[j] * q * pow(p[j], -q) * integral;
            if (re > cur) {
                d = re - cur;
                de += ekin_erg(p[j], s) * d * dp[j];
            }
        }
        dlt[j] = d;
    }
    return warp_sum(de);
}

// drury83 convolution (tracer_fp_dsa_reacc.c:105-161)
__device__ void reacc_convolution(const DsaArgs &A, int s, const double *N, double vup, double vdown,
                                  double q, double pmin, double *dlt, int lane)
{
    const double *p = A.p[s], *dp = A.dp[s];
    const double alpha = q - 2.0;
    double carry = 0.0;
    for (int j0 = 0; j0 < NB; j0 += 32) {
        const int j = j0 + lane;
        const bool use = j >= 1 && p[j] > 0.0 && p[j] >= pmin;
        const double seed = N[j * A.js] / vup, cur = N[j * A.js] / vdown;
        double term = 0.0;
        if (use) term = pow(p[j], alpha - 1.0) * seed * dp[j];
        const double incl = warp_scan(term, lane);
        const double integral = carry + incl;
        carry += __shfl_sync(kFull, incl, 31);
        double d = 0.0;
        if (use) {
            d = (alpha + 2.0) * pow(p[j], -alpha) * integral - cur;
            if (!isfinite(d)) d = 0.0;
            else if (d < -cur) d = -cur;
        }
        dlt[j] = d;
    }
}

__device__ double delta_edens(const DsaArgs &A, int s, const double *dlt, double pmin, int lane)
{
    const double *p = A.p[s], *dp = A.dp[s];
    double e = 0.0;
    for (int j = 2 + lane; j <= NB - 3; j += 32) {
        if (!(p[j] > 0.0) || p[j] < pmin || !isfinite(dlt[j])) continue;
        e += ekin_erg(p[j], s) * dlt[j] * dp[j];
    }
    return warp_sum(e);
}

// linear interpolation of N / vup at x over the bins [1, NB-2]
__device__ double interp_state(const double *p, const double *N, size_t js, double vup, double x)
{
    if (!(x > 0.0)) return 0.0;
    int lo = 1, hi = NB - 2;
    if (x < p[lo] || x > p[hi]) return 0.0;
    while (hi - lo > 1) {
        const int mid = lo + (hi - lo) / 2;
        if (p[mid] <= x) lo = mid;
        else hi = mid;
    }
    const double a = N[lo * js] / vup, b = N[hi * js] / vup;
    if (p[hi] <= p[lo]) return a;
    return a + (b - a) * (x - p[lo]) / (p[hi] - p[lo]);
}

// adiabatic compression delta (tracer_fp_dsa_reacc.c:187-236)
__device__ double reacc_adiabatic(const DsaArgs &A, int s, const double *N, double vup, double vdown,
                                  double ratio, double pmin, double *ad, int lane)
{
    const double *p = A.p[s];
    if (!(vup > 0.0) || !(vdown > 0.0) || !(ratio > 0.0) || !isfinite(ratio)) {
        for (int j = lane; j < NB; j += 32) ad[j] = 0.0;
        __syncwarp();
        return 0.0;
    }
    const double shift = cbrt(ratio), norm = shift * shift;
    for (int j = lane; j < NB; j += 32) {
        double d = 0.0;
        if (p[j] > 0.0 && p[j] >= pmin) {
            const double cur = N[j * A.js] / vdown;
            const double adv = norm * interp_state(p, N, A.js, vup, p[j] / shift);
            if (isfinite(cur) && isfinite(adv)) d = adv - cur;
        }
        ad[j] = d;
    }
    __syncwarp();
    return delta_edens(A, s, ad, pmin, lane);
}

__global__ void __launch_bounds__(kDsaWarps * 32) dsa_inject_kernel(DsaArgs A)
{
    extern __shared__ double4 smem_raw[];
    DsaSmem &sm = reinterpret_cast<DsaSmem *>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * kDsaWarps + (threadIdx.x >> 5);
    if (t >= A.ntracer) return;
    const CromaB200DsaParams &prm = A.prm;
    double mach, temp, rho1, u1;
    if (!resolve_input(A, t, mach, temp, rho1, u1)) return;
    const double ratio = compression_ratio(mach, prm.gamma_gas);
    if (!(ratio > 0.0) || !isfinite(ratio)) return;
    const double rho2 = ratio * rho1, u2 = u1 / ratio;
    double q = 0.0;
    if (mach > 1.0 && ratio > 1.0) q = 3.0 * ratio / (ratio - 1.0);
    if (!(q > 0.0) || !isfinite(q)) return;
    const double chi_e = (prm.chi_e > 0.0) ? prm.chi_e : prm.chi_p;
    const double pmin_p = injection_momentum(temp, prm.chi_p, kMpG);
    const double pmin_e = injection_momentum(temp, chi_e, kMeG);
    if (!(pmin_p > 0.0) || !isfinite(pmin_p) || !(pmin_e > 0.0) || !isfinite(pmin_e)) return;
    const int inj_p = prm.inject_species != 2, inj_e = prm.inject_species != 1;

    // fresh protons and electrons
    double A_p = 0.0, A_e = 0.0;
    const double eta = dsa_eta(mach, prm.eta_model_initial);
    if (mach > 1.0 && prm.gamma_gas > 1.0 && prm.chi_p > 0.0 && prm.pmax_p_mc > 0.0 && eta > 0.0 &&
        pmin_p < prm.pmax_p_mc) {
        const double unit = proton_edens_unit(pmin_p, q, prm.pmax_p_mc, lane);
        if (unit > 0.0 && rho1 > 0.0 && u1 > 0.0 && u2 > 0.0)
            A_p = eta * (0.5 * rho1 * u1 * u1 * u1) / u2 / unit;
    }
    const bool fresh_p = A_p > 0.0;
    if (fresh_p && inj_e && prm.pmax_e_mc > 0.0 && chi_e > 0.0 && pmin_e < prm.pmax_e_mc && prm.k_ep > 0.0) {
        const double mr = kMpG / kMeG;
        const double sp = spectrum_shape(pmin_p, pmin_p, q, prm.pmax_p_mc);
        const double se = spectrum_shape(mr * pmin_p, pmin_e, q, prm.pmax_e_mc);
        if (sp > 0.0 && se > 0.0) A_e = prm.k_ep * (1.0 / (mr * mr * mr)) * A_p * sp / se;
    }
    const bool fresh_e = A_e > 0.0;

    const double mass_g = A.mass[t] * kMsunG;
    const double vup = mass_g / rho1, vdown = mass_g / rho2;
    if (!(vup > 0.0) || !isfinite(vup) || !(vdown > 0.0) || !isfinite(vdown)) return;
    const double *Np = A.crp + (size_t)t * A.ts;
    const double *Ne = A.cre + (size_t)t * A.ts;

    // reacceleration deltas of the pre-shock spectra
    double scale = 0.0, energy = 0.0;
    const bool reacc = A.reacc == 1 || A.reacc == 2;
    if (reacc) {
        for (int j = lane; j < NB; j += 32) {
            sm.dlt[0][j] = 0.0;
            sm.dlt[1][j] = 0.0;
        }
        __syncwarp();
    }
    if (A.reacc == 1) {
        // X_cr = P_cr / P_th with E_cr above xcr_pmin (tracer_dsa_xcr_proton)
        double e = 0.0;
        for (int j = lane; j < NB; j += 32)
            if (A.p[0][j] >= prm.xcr_pmin_pmc) e += ekin_erg(A.p[0][j], 0) * Np[j * A.js] * A.dp[0][j];
        const double ecr = warp_sum(e) / vdown;
        const double pth = rho1 * kKbCgs * temp / (prm.mu_mol * kMpG);
        double xcr = 0.0;
        if (pth > 0.0 && isfinite(ecr / 3.0) && isfinite(pth) && ecr / 3.0 > 0.0) xcr = (ecr / 3.0) / pth;
        double eta_int = 0.0;
        const int ii = prm.eta_model_initial, ir = prm.eta_model_reacc;
        if (ii >= 0 && ii < 8 && ir >= 0 && ir < 8) {
            const double ei = dsa_eta(mach, ii), er = dsa_eta(mach, ir);
            const double x0 = c_models[ir].xcr0;
            if (x0 <= 0.0) {
                eta_int = ei;
            } else {
                const double wgt = fmin(fmax(xcr / x0, 0.0), 1.0);
                eta_int = (1.0 - wgt) * ei + wgt * er;
            }
        }
        double extra = eta_int - dsa_eta(mach, ii);
        if (extra < 0.0 || !isfinite(extra)) extra = 0.0;
        const double budget = extra * 0.5 * mass_g * u1 * u1;
        if (budget > 0.0) {
            const double ep = reacc_positive(A, 0, Np, vdown, q, pmin_p, sm.dlt[0], lane);
            const double ee = reacc_positive(A, 1, Ne, vdown, q, pmin_e, sm.dlt[1], lane);
            energy = (ep + ee) * vdown;
            if (energy > 0.0 && isfinite(energy)) {
                scale = (energy > budget) ? budget / energy : 1.0;
            } else {
                __syncwarp();
                for (int j = lane; j < NB; j += 32) {
                    sm.dlt[0][j] = 0.0;
                    sm.dlt[1][j] = 0.0;
                }
            }
        }
        __syncwarp();
    } else if (A.reacc == 2) {
        reacc_convolution(A, 0, Np, vup, vdown, q, pmin_p, sm.dlt[0], lane);
        reacc_convolution(A, 1, Ne, vup, vdown, q, pmin_e, sm.dlt[1], lane);
        __syncwarp();
        const double cp = delta_edens(A, 0, sm.dlt[0], pmin_p, lane);
        const double ce = delta_edens(A, 1, sm.dlt[1], pmin_e, lane);
        energy = (cp + ce) * vdown;
        scale = 1.0;
        if (prm.reacc_eta_cap > 0.0 && isfinite(prm.reacc_eta_cap)) {
            const double budget = prm.reacc_eta_cap * 0.5 * mass_g * u1 * u1;
            const double ap = reacc_adiabatic(A, 0, Np, vup, vdown, ratio, pmin_p, sm.ad[0], lane);
            const double ae = reacc_adiabatic(A, 1, Ne, vup, vdown, ratio, pmin_e, sm.ad[1], lane);
            const double nonad = (cp + ce - ap - ae) * vdown;
            if (nonad > 0.0 && isfinite(nonad) && budget > 0.0 && isfinite(budget)) {
                if (nonad > budget) scale = budget / nonad;
                for (int j = lane; j < NB; j += 32) {
                    sm.dlt[0][j] = sm.ad[0][j] + scale * (sm.dlt[0][j] - sm.ad[0][j]);
                    sm.dlt[1][j] = sm.ad[1][j] + scale * (sm.dlt[1][j] - sm.ad[1][j]);
                }
                energy = (ap + ae + scale * (cp + ce - ap - ae)) * vdown;
            }
        }
        __syncwarp();
        if (A.dis && lane == 0) A.dis[t] = 1;
    }

    // apply: fresh sources, then the reacceleration deltas (from the
    // pre-shock spectra read above)
    const bool state = A.mode == 1;
    double *Op = state ? A.crp + (size_t)t * A.ts : A.qpi + (size_t)t * A.ts;
    double *Oe = state ? A.cre + (size_t)t * A.ts : A.qepri + (size_t)t * A.ts;
    const double inv_dt = state ? 1.0 : 1.0 / A.dt_gyr;
    const double s_re = (A.reacc == 2) ? 1.0 : scale;
    const double *gp = A.dsa_p, *ge = A.dsa_p + NB;
    for (int j = lane; j < NB; j += 32) {
        double vp = Op[j * A.js], ve = Oe[j * A.js];
        if (inj_p && fresh_p) {
            const double src = source_dp(A_p, pmin_p, q, prm.pmax_p_mc, gp[j]);
            vp += state ? src * vdown : src * vdown * inv_dt;
        }
        if (inj_e && fresh_p && fresh_e) {
            const double src = source_dp(A_e, pmin_e, q, prm.pmax_e_mc, ge[j]);
            ve += state ? src * vdown : src * vdown * inv_dt;
        }
        if (reacc) {
            vp += state ? sm.dlt[0][j] * vdown * s_re : sm.dlt[0][j] * vdown * s_re * inv_dt;
            ve += state ? sm.dlt[1][j] * vdown * s_re : sm.dlt[1][j] * vdown * s_re * inv_dt;
        }
        Op[j * A.js] = vp;
        Oe[j * A.js] = ve;
    }
    bool applied = (inj_p && fresh_p) || (inj_e && fresh_p && fresh_e);
    if (reacc && scale > 0.0 && isfinite(energy) && fabs(energy) > 0.0) applied = true;
    if (applied && lane == 0) atomicAdd(A.count, 1u);
}

}  // namespace

int dsa_inject(Context &c, const CromaB200Shocks *sh, double density_unit, double dt_gyr, int mode,
               int reacc_mode, int *ninjected)
{
    if (ninjected) *ninjected = 0;
    if (mode == 0) return 0;
    if (mode != 1 && mode != 2) { set_error("unknown DSA injection mode"); return -1; }
    if (reacc_mode < 0 || reacc_mode > 2) { set_error("unknown DSA reacceleration mode"); return -1; }
    if (mode == 2 && (!(dt_gyr > 0.0) || !isfinite(dt_gyr))) {
        set_error("tracer_source DSA injection needs dt_gyr > 0");
        return -1;
    }
    if (!c.dsa_set || !c.d_dsa_p) { set_error("croma_b200_set_dsa must come first"); return -1; }
    if (c.cap <= 0) { set_error("reserve/set_state before DSA injection"); return -1; }
    const int n = c.cap;
    // shock fields to the device
    const double *src[10] = {sh->mach, sh->prestemp, sh->presden, sh->pre_density_cgs,
                             sh->upstream_speed_cgs, sh->shock_side_code, sh->dsa_trigger,
                             sh->dsa_mach, sh->dsa_pre_density, sh->dsa_flux_cgs};
    const double *dev[10];
    if (sh->on_device) {
        for (int k = 0; k < 10; k++) dev[k] = src[k];
    } else {
        if (c.dsa_stage_cap < n) {
            dev_free(c, c.d_dsa_stage);
            c.d_dsa_stage = nullptr;
            c.dsa_stage_cap = 0;
            CROMA_CUDA(dev_alloc(c, &c.d_dsa_stage, (size_t)10 * n * sizeof(double)));
            c.dsa_stage_cap = n;
        }
        for (int k = 0; k < 10; k++) {
            dev[k] = nullptr;
            if (!src[k]) continue;
            double *d = c.d_dsa_stage + (size_t)k * n;
            CROMA_CUDA(cudaMemcpyAsync(d, src[k], (size_t)n * sizeof(double), cudaMemcpyHostToDevice,
                                       c.stream));
            dev[k] = d;
        }
    }
    DsaArgs A{};
    A.prm = c.dsa;
    A.mach = dev[0]; A.prestemp = dev[1]; A.presden = dev[2]; A.pre_density_cgs = dev[3];
    A.upstream_speed_cgs = dev[4]; A.shock_side_code = dev[5]; A.dsa_trigger = dev[6];
    A.dsa_mach = dev[7]; A.dsa_pre_density = dev[8]; A.dsa_flux = dev[9];
    A.has_dsa = sh->has_dsa;
    A.ntracer = n;
    A.density_unit = density_unit;
    A.dt_gyr = dt_gyr;
    A.mode = mode;
    A.reacc = reacc_mode;
    A.crp = c.d_crp;
    A.cre = c.d_cre;
    A.qpi = c.d_qpi;
    A.qepri = c.d_qepri;
    A.ts = NB;   // cell-major [tracer][nb]
    A.js = 1;
    A.dis = c.d_dis;
    A.mass = c.d_mass;
    for (int s = 0; s < 2; s++) { A.p[s] = c.gt.s[s].p; A.dp[s] = c.gt.s[s].dp; }
    A.dsa_p = c.d_dsa_p;
    A.count = c.d_dsa_count;
    // per snapshot, as the reference's snapshot driver does: the sources of
    // tracer_source mode and the disable-adiabatic flags start from zero
    const size_t st = (size_t)NB * n * sizeof(double);
    if (mode == 2) {
        CROMA_CUDA(cudaMemsetAsync(c.d_qpi, 0, st, c.stream));
        CROMA_CUDA(cudaMemsetAsync(c.d_qepri, 0, st, c.stream));
        c.has_sources = 1;
    }
    CROMA_CUDA(cudaMemsetAsync(c.d_dis, 0, (size_t)n, c.stream));
    CROMA_CUDA(cudaMemsetAsync(c.d_dsa_count, 0, sizeof(unsigned), c.stream));
    constexpr size_t smem = kDsaWarps * sizeof(DsaSmem);
    // set once per process; thread-safe (function-local static initialisation)
    static const cudaError_t attr =
        cudaFuncSetAttribute(dsa_inject_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    CROMA_CUDA(attr);
    dsa_inject_kernel<<<(n + kDsaWarps - 1) / kDsaWarps, kDsaWarps * 32, smem, c.stream>>>(A);
    CROMA_CUDA(cudaGetLastError());
    c.last_launches += 1;
    unsigned cnt = 0;
    CROMA_CUDA(cudaMemcpyAsync(&cnt, c.d_dsa_count, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    if (ninjected) *ninjected = (int)cnt;
    // The reference always evolves both species (src/tracer_fp_cpu.c:149-190);
    // a species left out of the mask is skipped only while its spectra and
    // sources are zero, so a species that received particles joins the mask.
    if (cnt > 0) {
        int add = 0;
        if (c.dsa.inject_species != 1 || reacc_mode != 0) add |= CROMA_SPECIES_PROTON;
        if (c.dsa.inject_species != 2 || reacc_mode != 0) add |= CROMA_SPECIES_ELECTRON;
        c.mp.species_mask |= add;
        c.cfg.species_mask |= add;
    }
    return 0;
}

// DSA-grid momenta at the FP bins (dsa_init_grid, src/DSA_MODELS.c:1191-1261):
// the grid extends the FP grid's log spacing down to pmin_dsa and recomputes
// p = 10^(pmin + j dlogp); FP bin j is DSA bin j + n_extra.
int set_dsa(Context &c, const CromaB200DsaParams *prm)
{
    if (!prm) { set_error("null DSA parameters"); return -1; }
    if (prm->eta_model_initial < 0 || prm->eta_model_initial > 7 || prm->eta_model_reacc < 0 ||
        prm->eta_model_reacc > 7) {
        set_error("DSA efficiency model id out of range (0..7)");
        return -1;
    }
    std::vector<double> h(2 * NB);
    const double lim[2] = {prm->pmin_dsa_p_log10, prm->pmin_dsa_e_log10};
    for (int s = 0; s < 2; s++) {
        const std::vector<double> &p = c.h_p[s];
        if ((int)p.size() < 2 || !(p[0] > 0.0)) { set_error("grid not built"); return -1; }
        const double dlogp = log10(p[1]) - log10(p[0]);
        const double pmin_fp = log10(p[0]);
        int extra = 0;
        if (dlogp > 0.0 && lim[s] < pmin_fp) {
            extra = (int)ceil((pmin_fp - lim[s]) / dlogp - 1.0e-12);
            if (extra < 0) extra = 0;
        }
        const double base = pmin_fp - dlogp * (double)extra;
        for (int j = 0; j < NB; j++) h[(size_t)s * NB + j] = pow(10.0, base + dlogp * (double)(j + extra));
    }
    if (!c.d_dsa_p) {
        CROMA_CUDA(dev_alloc(c, &c.d_dsa_p, 2 * NB * sizeof(double)));
        CROMA_CUDA(dev_alloc(c, &c.d_dsa_count, sizeof(unsigned)));
    }
    CROMA_CUDA(cudaMemcpyAsync(c.d_dsa_p, h.data(), 2 * NB * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    c.dsa = *prm;
    c.dsa_set = 1;
    return 0;
}

void free_dsa(Context &c)
{
    dev_free(c, c.d_dsa_p);
    dev_free(c, c.d_dsa_count);
    dev_free(c, c.d_dsa_stage);
    c.d_dsa_p = c.d_dsa_stage = nullptr;
    c.d_dsa_count = nullptr;
    c.dsa_stage_cap = 0;
    c.dsa_set = 0;
}

}  // namespace croma
