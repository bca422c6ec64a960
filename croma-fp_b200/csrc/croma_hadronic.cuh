// croma_hadronic.cuh -- hadronic (pp) pieces of the tracer update:
// the Kamae (2006) pion production cross section used for the proton
// catastrophic-loss time, and the secondary-electron production kernel
// (Brunetti & Blasi 2005 with the Kelner (2006) pion spectrum) that feeds
// the secondary electron source.  Restated from src/HADRONIC.c of
// kosukenishiwaki/croma-fp; parameter tables are Kamae (2006, errata 2007),
// Blattnig (2000) and Kelner (2006) as used there.
#pragma once

#include "croma_phys.cuh"

namespace croma {

// pp_pion_cross_section, src/HADRONIC.c:342-429 (p in GeV/c).
CROMA_HD double pp_pion_xsec(int kind, double p)
{
    const double a0 = 0.1176, a1 = 0.3829, a2 = 23.10, a3 = 6.454, a4 = -5.764,
                 a5 = -23.63, a6 = 94.75, a7 = 0.02667;
    const double b0 = 11.34, b1 = 23.72;
    const double c0 = 28.5, c1 = -6.133, c2 = 1.464;
    const double d0 = 0.3522, d1 = 0.1530, d2 = 1.498, d3 = 2.0, d4 = 30.0, d5 = 3.155, d6 = 1.042;
    const double e0 = 5.922, e1 = 1.632;
    const double f0 = 0.0834, f1 = 9.5, f2 = 5.5, f3 = 1.68, f4 = 3134.0;
    const double g0 = 0.0004257, g1 = 4.5, g2 = 7.0, g3 = 2.1, g4 = 503.5;
    if (kind > 2 || kind < -2) return 0.0;
    const double Ep = sqrt(kMp * kMp + p * p), Tp = Ep - kMp;
    const double x = log10(p), x2 = x * x, x3 = x2 * x;
    double nondiff, diff, dres, res;

    if (p < 1.0) nondiff = 0.0;
    else if (p < 1.3) nondiff = 0.57 * pow(x / a0, 1.2) * (a2 + a3 * x2 + a4 * x3 + a5 * exp(-a6 * pow(x + a7, 2.0)));
    else if (p < 2.4) nondiff = (b0 * fabs(a1 - x) + b1 * fabs(a0 - x)) / (a1 - a0);
    else if (p < 10.0) nondiff = a2 + a3 * x2 + a4 * x3 + a5 * exp(-a6 * pow(x + a7, 2.0));
    else nondiff = c0 + c1 * x + c2 * x2;

    if (p < 2.25) diff = 0.0;
    else if (p < 3.2) diff = sqrt(fabs(x - d0) / d1) * (d2 + d3 * log10(d4 * (x - 0.25)) + d5 * x2 - d6 * x3);
    else if (p < 100.0) diff = d2 + d3 * log10(d4 * (x - 0.25)) + d5 * x2 - d6 * x3;
    else diff = e0 + e1 * x;

    if (Ep < 1.4) dres = 0.0;
    else if (Ep < 1.6) dres = f0 * pow(Ep, 10.0);
    else if (Ep < 1.8) dres = f1 * exp(-f2 * pow(Ep - f3, 2.0));
    else if (Ep < 10.0) dres = f4 * pow(Ep, -10.0);
    else dres = 0.0;

    if (Ep < 1.6) res = 0.0;
    else if (Ep < 1.9) res = g0 * pow(Ep, 14.0);
    else if (Ep < 2.3) res = g1 * exp(-g2 * pow(Ep - g3, 2.0));
    else if (Ep < 20.0) res = g4 * pow(Ep, -6.0);
    else res = 0.0;

    const double tot = (nondiff + diff + dres + res) * kMb;
    const double r0 = 1.0 / (0.007 + 0.1 * log(Tp) / Tp + 0.3 / Tp / Tp);
    const double rp = 1.0 / (0.00717 + 0.0652 * log(Tp) / Tp + 0.162 / Tp / Tp);
    const double rm = 1.0 / (0.00456 + 0.0846 / pow(Tp, 0.5) + 0.577 / pow(Tp, 1.5));
    if (kind == 0) return tot;
    if (kind == 1) return tot * rp / r0;
    if (kind == -1) return tot * rm / r0;
    return tot * (1.0 + rp / r0 + rm / r0);
}

// FpiQ, src/HADRONIC.c:324-336 (Kelner QGSJET pion spectrum).
CROMA_HD double fpi_q(int m, double Epi, double Ep)
{
    const double L = log(0.001 * Ep), x = Epi / Ep;
    const double mpi = (m == 1) ? 1.40e-1 : 1.35e-1;
    if (x <= mpi / Ep) return 0.0;
    if (x > 1.0) return 0.0;
    const double Bpi = 5.58 + 0.78 * L + 0.10 * L * L;
    const double alpha = 0.89 / (sqrt(Bpi) * (1.0 - exp(-0.33 * Bpi)));
    const double r = 3.1 / (pow(Bpi, 1.5));
    const double xa = pow(x, alpha);
    double A = pow((1.0 - xa) / pow(1.0 + r * xa, 3.0), 4.0);
    A = A * (1.0 / (1.0 - xa) + 3.0 * r / (1.0 + r * xa)) * sqrt(1.0 - mpi / (x * Ep));
    return 4.0 * alpha * Bpi * xa * A / x / Ep;
}

CROMA_HD double dsigma(int i, double Epi, double Ep)   // src/HADRONIC.c:291-300
{
    const double gp = Ep / kMp, gbp = sqrt(gp * gp - 1.0), pp = gbp * kMp;
    const double Fpi = fpi_q(0, Epi, Ep);
    const double s = pp_pion_xsec(i, pp);
    return s * Fpi / sqrt(1.0 + 1.0 / (gbp * gbp));
}

CROMA_HD double lorentz_beta(double gamma)              // src/HADRONIC.c:431-435
{
    const double b2 = gamma * gamma - 1.0;
    if (b2 < 0.0) return 0.0;
    return sqrt(b2) / gamma;
}

CROMA_HD double fe_bl10(double Ee, double Epi)          // Fe, src/HADRONIC.c:499-533
{
    const double mpi = 1.3957e-1, mmu = 1.05658e-1, bmu = 0.2714;
    const double gpi = Epi / mpi;
    const double xi = mmu * mmu / (mpi * mpi);
    const double Emu = (mpi * mpi - mmu * mmu) / (mpi * mpi) * Epi / (2.0 * bmu);
    const double betamu = sqrt(1.0 - mmu * mmu / (Emu * Emu));
    const double lambda = 2.0 * mpi * mpi * Ee * bmu / ((mpi * mpi - mmu * mmu) * Epi);
    const double l2 = lambda * lambda, l3 = l2 * lambda;
    const double P = 1.0 / betamu * (2.0 * Epi * xi / (Emu * (1.0 - xi)) - (1.0 + xi) / (1.0 - xi));
    if (lambda > 1.0) return 0.0;
    if (gpi == 1.0) return 0.0;
    if (lambda < 0.0) return 0.0;
    const double om = 1.0 - betamu;
    if (om / (1.0 + betamu) < lambda) {
        const double X = 5.0 - 9.0 * l2 + 4.0 * l3 -
                         P / betamu * (1.0 - (6.0 * betamu + 3.0) * l2 + (6.0 * betamu + 2.0) * l3);
        return X / 12.0;
    } else if (lambda < om / (1.0 + betamu)) {
        return l2 * betamu / (om * om) * (3.0 - 2.0 / 3.0 * lambda * (3.0 + betamu * betamu) / om) -
               P / om * (l2 * (1.0 + betamu) - 2.0 * l2 / om * (0.5 + lambda * (1.0 + betamu)) +
                         2.0 * l3 * (3.0 + betamu * betamu) / (3.0 * (om * om)));
    }
    return 0.0;
}

// QeKernel_BB05, src/HADRONIC.c:436-497.  Constants of include/HADRONIC.h:
// threshold 0.289 GeV, log-E step 0.05, at least 50 steps.
CROMA_HD double qe_kernel(double Ee, double p)
{
    const double bmu = 0.2714;
    const double gp = sqrt(p * p + 1.0), Ep = gp * kMp, Emax = gp * kMp;
    const double r = 0.5 * (kMpiCh * kMpiCh - kMmu * kMmu) / (bmu * kMpiCh * kMpiCh);
    double Emin = Ee / r;
    if (Emax < Emin || (Ep - kMp) < 0.289) return 0.0;
    Emin = fmax(Emin, kMpiCh);
    const double da = 0.05;
    const double amin = log10(Emin), amax = log10(Emax);
    const int Na = (int)fmax(50.0, round((amax - amin) / da));
    double a = amin, Epi = pow(10.0, a), integral = 0.0, f;
    double betamu = lorentz_beta(Epi * r / kMmu);
    if (betamu == 0.0) f = 0.0;
    else f = (dsigma(1, Epi, Ep) + dsigma(-1, Epi, Ep)) * fe_bl10(Ee, Epi) / (betamu * Epi);
    for (int i = 1; i < Na; i++) {
        const double Epipre = Epi;
        a = a + da;
        Epi = pow(10.0, a);
        const double dEpi = Epi - Epipre;
        const double fpre = f;
        betamu = lorentz_beta(Epi * r / kMmu);
        f = (dsigma(1, Epi, Ep) + dsigma(-1, Epi, Ep)) * fe_bl10(Ee, Epi) / (betamu * Epi);
        integral = integral + 0.5 * (f + fpre) * dEpi;
        if (integral < 0.0 || isnan(integral)) return 0.0;
    }
    return 8.0 * bmu * kMpiCh * kMpiCh * (kC * kMe) * integral / (kMpiCh * kMpiCh - kMmu * kMmu);
}

// ----------------------------------------------------------------------
// Emission kernels of the pp interaction (the gamma and neutrino tables of
// prepare_gamma_kernel_flat / prepare_neutrino_kernel_flat,
// src/fp_shared_core.c:1724-1778).  Kelner (2006) energy distributions over
// the same pion spectrum and cross sections as the secondaries above; the
// step counts are include/HADRONIC.h:6-12 (200 pion-energy / x steps,
// thresholds 0.285 / 0.289 / 0.29 GeV).
// ----------------------------------------------------------------------
constexpr double kMpi0 = 1.35e-1;          // pion0_mass_gev, src/CONSTANTS.c:21
constexpr int kHadronSteps = 200;          // HADRON_KERNEL_EPI_STEPS = HADRON_ELECTRON_X_STEPS

// gammaKernel, src/HADRONIC.c:139-177: pi0 -> 2 gamma, trapezoid over a
// log-spaced pion energy from E_g + m_pi0^2 / (4 E_g) to E_p.
CROMA_HD double gamma_kernel(double Eg, double p)
{
    const double gp = sqrt(p * p + 1.0), Ep = gp * kMp;
    const double Emax = Ep;
    double Emin = Eg + kMpi0 * kMpi0 / (4.0 * Eg);
    if (Emax < Emin) return 0.0;
    if (Emin < kMpi0) Emin = kMpi0;
    if ((Ep - kMp) < 0.285) return 0.0;
    const double amin = log10(Emin), amax = log10(Emax), da = (amax - amin) / (double)kHadronSteps;
    double a = amin, Epi = pow(10.0, a);
    double f = dsigma(0, Epi, Ep) / sqrt(Epi * Epi - kMpi0 * kMpi0), integral = 0.0;
    for (int i = 1; i < kHadronSteps; i++) {
        const double Epipre = Epi, fpre = f;
        a += da;
        Epi = pow(10.0, a);
        const double dEpi = Epi - Epipre;
        f = dsigma(0, Epi, Ep) / sqrt(Epi * Epi - kMpi0 * kMpi0);
        integral += 0.5 * (f + fpre) * dEpi;
    }
    return 2.0 * kC * integral / (4.0 * kPi);
}

// Kelner (2006) eq. (36): electron / muon-neutrino spectrum from muon decay
// in the pion frame (fe, src/HADRONIC.c:302-310).
CROMA_HD double kelner_fe(double x)
{
    const double r = kMmu * kMmu / (kMpiCh * kMpiCh), x2 = x * x, r2 = r * r;
    if (x > r) return (3.0 - 2.0 * r) * (9.0 * x2 - 6.0 * log(x) - 4.0 * x2 * x - 5.0) / (9.0 * pow(1.0 - r, 2.0));
    const double h1 = (3.0 - 2.0 * r) * (9.0 * r2 - 6.0 * log(r) - 4.0 * r2 * r - 5.0) / (9.0 * pow(1.0 - r, 2.0));
    const double h2 = (1.0 + 2.0 * r) * (r - x) * (9.0 * (r + x) - 4.0 * (r2 + r * x + x2)) / (9.0 * r2);
    return h1 + h2;
}

// Kelner (2006) eq. (40): electron-neutrino spectrum, r = 0.573
// (fnue, src/HADRONIC.c:311-320).
CROMA_HD double kelner_fnue(double x)
{
    const double r = 0.573, x2 = x * x, r2 = r * r;
    if (x > r)
        return 2.0 * (1.0 - x) * (6.0 * pow(1.0 - x, 2.0) + r * (5.0 + 5.0 * x - 4.0 * x2) + 6.0 * r * log(x) / (1.0 - x)) /
               (3.0 * pow(1.0 - r, 2.0));
    const double h1 = 2.0 * ((1.0 - r) * (6.0 - 7.0 * r + 11.0 * r2 - 4.0 * r2 * r) + 6.0 * r * log(r)) /
                      (3.0 * pow(1.0 - r, 2.0));
    const double h2 = 2.0 * (r - x) * (7.0 * r2 - 4.0 * r2 * r + 7.0 * x * r - 4.0 * x * r2 - 2.0 * x2 - 4.0 * x2 * r) /
                      (3.0 * r2);
    return h1 + h2;
}

enum LeptonKind { kLeptonElectron = 0, kLeptonNue = 1, kLeptonNumu = 2 };   // HadronLeptonKernel

// One charge of eKernel's sum: trapezoid in x = E / E_pi on (0, 1) with the
// first interval taken as a rectangle (src/HADRONIC.c:200-236).
template <int KIND>
CROMA_HD double lepton_x_integral(int charge, double E, double Ep)
{
    const double dx = 1.0 / (double)kHadronSteps;
    double x = 0.0, f = 0.0, integral = 0.0;
    for (int i = 1; i < kHadronSteps; i++) {
        x += dx;
        const double Epi = E / x, fpre = f;
        f = dsigma(charge, Epi, Ep) * (KIND == kLeptonNue ? kelner_fnue(x) : kelner_fe(x)) / x;
        integral += (i == 1) ? f * dx : 0.5 * (f + fpre) * dx;
    }
    return integral;
}

// eKernel, src/HADRONIC.c:181-236, for the neutrino kinds (the electron kind
// is the secondary source, qe_kernel above).
template <int KIND>
CROMA_HD double lepton_kernel(double E, double p)
{
    const double gp = sqrt(p * p + 1.0), Ep = gp * kMp;
    const double Emax = gp * kMp;
    const double Emin = 2.0 * E * kMpiCh * kMpiCh / (kMpiCh * kMpiCh + kMmu * kMmu);
    if (Emax < Emin) return 0.0;
    if ((Ep - kMp) < 0.289) return 0.0;
    const double i1 = lepton_x_integral<KIND>(1, E, Ep);
    const double i2 = lepton_x_integral<KIND>(-1, E, Ep);
    return kC * (i1 + i2) / (4.0 * kPi);
}

// numu1Kernel, src/HADRONIC.c:240-289: muon neutrinos of the pion decay
// itself, x = E / E_pi on (0, lambda).
CROMA_HD double numu_pion_kernel(double Enu, double p)
{
    const double lambda = 1.0 - kMmu * kMmu / (kMpiCh * kMpiCh);
    const double gp = sqrt(p * p + 1.0), Ep = gp * kMp, Emax = gp * kMp, Emin = Enu / lambda;
    if (Emax < Emin) return 0.0;
    if ((Ep - kMp) < 0.29) return 0.0;
    const double dx = lambda / (double)kHadronSteps;
    double sum[2];
    for (int s = 0; s < 2; s++) {
        const int charge = s ? -1 : 1;
        double x = 0.0, f = 0.0, integral = 0.0;
        for (int i = 1; i < kHadronSteps; i++) {
            x += dx;
            const double Epi = Enu / x, fpre = f;
            f = dsigma(charge, Epi, Ep) / x;
            integral += (i == 1) ? f * dx : 0.5 * (f + fpre) * dx;
        }
        sum[s] = integral;
    }
    return kC * (sum[0] + sum[1]) / lambda / (4.0 * kPi);
}

// One entry of the neutrino table: muon + electron neutrinos of muon decay
// plus the muon neutrino of the pion decay (prepare_neutrino_kernel_flat,
// src/fp_shared_core.c:1771-1773, in that order).
CROMA_HD double neutrino_kernel(double Enu, double p)
{
    return lepton_kernel<kLeptonNumu>(Enu, p) + lepton_kernel<kLeptonNue>(Enu, p) + numu_pion_kernel(Enu, p);
}

}  // namespace croma
