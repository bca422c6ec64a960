/* Test infrastructure, not product code: the CPU restatement of the
 * per-tracer background preparation that the checks compare the device
 * kernel (croma_b200_background_prepare) with.
 *
 * or_background restates, over arrays of tracers:
 *   the raw unit scaling of tracer_load_hdf5_raw_snapshot_slice
 *     (src/tracer_fp_background.c:1189-1197): density * c_dens, B * c_mag;
 *   tracer_prepare_background_from_raw (:1206-1263): div v * Gyr, curl v,
 *     target scale L_turb_target_kpc * kpc (:1216, :37);
 *   prepare_background_cell (src/fp_shared_core.c:866-932) with c_sound
 *     (src/FP_Coef.c:916-919), dv_limit (:622-628), B_dynamo (:929-931);
 *   tracer_store_background_history_slot (src/tracer_fp_background.c:324-342):
 *     the eight stored fields, field-major bg[8][n].
 * Expressions keep the reference's evaluation order, so that gcc gives the
 * same roundings (pinned to the compiled reference in
 * tests/test_histories.py). */
#include <math.h>
#include <stddef.h>

#include "croma_oracle.h"

int or_background(int n, const double *temp_K, const double *density, const double *bx, const double *by,
                  const double *bz, const double *div_v, const double *curl_prev, const double *curl,
                  const double *curl_next, const double *l_turb_cm, double c_dens, double c_mag, double z_prev,
                  double z_curr, double z_next, int apply_temp_floor, int allow_curl_interp, int bfield_mode,
                  double mu_mol, double eta_B, double mach_limit, double l_turb_target_kpc, double *bg)
{
    const double kB = 8.62e-5, c = 2.999e+10, eV = 1.6e-12, Mpc = 3.0857e+24;
    const double kpc = 3.0857e21, gyr = 3.1536e16;
    const double target = l_turb_target_kpc * kpc;
    int bad = 0;
    for (int i = 0; i < n; i++) {
        const double rho = density[i] * c_dens;
        const double bxg = bx[i] * c_mag, byg = by[i] * c_mag, bzg = bz[i] * c_mag;
        const double divv_gyr = 1.0 * div_v[i] * gyr;
        double t = temp_K[i], cv = 1.0 * curl[i];
        if (rho <= 0.0 || target <= 0.0) {
            bad = 1;
            for (int f = 0; f < 8; f++) bg[(size_t)f * n + i] = 0.0;
            continue;
        }
        if (apply_temp_floor && t < 1.0e4) t = 1.0e4;
        if (allow_curl_interp && cv == 0.0 && z_next != z_prev) {
            const double cp = 1.0 * curl_prev[i], cn = 1.0 * curl_next[i];
            cv = (cn - cp) / (z_next - z_prev) * (z_curr - z_prev) + cp;
        }
        double lt = (l_turb_cm && l_turb_cm[i] > 0.0) ? l_turb_cm[i] : target;
        double dv = cv * lt;
        const double cs = sqrt(5.0 / 3.0 * kB * t / (mu_mol * 0.938 * 1.0e+9)) * c;
        dv *= pow(target / lt, 0.3333);
        lt = target;
        if (mach_limit > 0.0 && cs > 0.0 && dv / cs > mach_limit) dv = mach_limit * cs;
        const double b_sim = sqrt(bxg * bxg + byg * byg + bzg * bzg);
        const double b_dyn = sqrt(4.0 * M_PI * eta_B * rho * dv * dv);
        const double b_eff = bfield_mode == 1 ? b_sim : (bfield_mode == 2 ? b_dyn : fmax(b_dyn, b_sim));
        const double n_gas = rho / (1.6e-24 * mu_mol);
        const double beta = b_eff > 0.0 ? n_gas * kB * t * eV / (b_eff * b_eff / (8.0 * M_PI)) : 1.0e10;
        bg[0 * (size_t)n + i] = n_gas;
        bg[1 * (size_t)n + i] = kB * t * 1.0e-9;
        bg[2 * (size_t)n + i] = b_eff;
        bg[3 * (size_t)n + i] = divv_gyr;
        bg[4 * (size_t)n + i] = lt / Mpc;
        bg[5 * (size_t)n + i] = dv;
        bg[6 * (size_t)n + i] = cs;
        bg[7 * (size_t)n + i] = beta;
    }
    return bad ? -2 : 0;
}
