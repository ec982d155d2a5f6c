// Monin-Obukhov surface-layer relations of the Schumann-Grotzbach wall
// functions (wallfunctions.c:12-290), device side: uStarShumann (friction
// velocity for a given wall heat flux) and qWallShumann (heat flux and
// friction velocity for a temperature difference between the first cell and
// the surface). Both iterate with under-relaxation 0.5 to a change below
// 1e-5 or 500 sweeps (then the neutral values), clamp |L| >= 1e-10, cap the
// unstable zeta at -1/15 + 1e-8 with the Businger-Dyer psi functions, and
// replace a stable result with u* < 1e-2 (no root) by the u* of a bisection
// on the slope of U_model(u*) (at most 50 halvings of [1e-6, u*_neutral]).
// The steps are the reference's, so that the sweep at which the iteration
// stops, and with it the result, is the same. A wall distance not above the
// roughness (a fatal error of the reference) returns NaN.
#pragma once
#include <cmath>

namespace tg {

namespace mo {

constexpr double kG = 9.81, kTol = 1e-5, kOmega = 0.5;
constexpr int kIterMax = 500;

__device__ __forceinline__ double clamp_l(double L) { return (L > 0) ? fmax(1e-10, L) : fmin(-1e-10, L); }

// psiM, psiH at zeta = z/L (stable: linear; unstable: Businger-Dyer)
__device__ __forceinline__ void psi(double zeta, bool stable, double gammaM, double gammaH, double &psiM, double &psiH)
{
    if (stable) { psiM = -gammaM * zeta; psiH = -gammaH * zeta; return; }
    if (zeta < -1.0 / 15.0) zeta = -1.0 / 15.0 + 1e-8;
    const double xi = pow(1.0 - 15.0 * zeta, 0.25);
    psiM = 2.0 * log((1.0 + xi) / 2.0) + log((1.0 + xi * xi) / 2.0) - 2.0 * atan(xi) + M_PI / 2.0;
    psiH = 2.0 * log((1.0 + xi * xi) / 2.0);
}

__device__ __forceinline__ double stable_slope(double u, double U, double wallDist, double z0, double gammaM, double kappa,
                                               double q, double thetaRef)
{
    const double Lq = fmax(1e-10, -pow(u, 3.0) / (kappa * (kG / thetaRef) * q));
    const double psiM = -gammaM * (wallDist / Lq);
    return ((u / kappa) * (log(wallDist / z0) - psiM) - U) / u;
}

__device__ __forceinline__ double stable_bisection(double U, double wallDist, double z0, double gammaM, double kappa, double q,
                                                   double thetaRef, double uNeutral)
{
    double uLow = 1e-6, uHigh = uNeutral, uMid = 0.0;
    for (int it = 0; it < 50; it++) {
        uMid = 0.5 * (uLow + uHigh);
        const double dfMid = stable_slope(uMid, U, wallDist, z0, gammaM, kappa, q, thetaRef);
        if (fabs(uHigh - uLow) < 1e-6 || fabs(dfMid) < kTol) break;
        const double dfLow = stable_slope(uLow, U, wallDist, z0, gammaM, kappa, q, thetaRef);
        if ((dfLow > 0 && dfMid > 0) || (dfLow < 0 && dfMid < 0)) uLow = uMid;
        else uHigh = uMid;
    }
    return uMid;
}

// uStarShumann, wallfunctions.c:12-130
__device__ __forceinline__ double ustar(double U, double wallDist, double z0, double gammaM, double kappa, double qwall,
                                        double thetaRef)
{
    if (!(wallDist > z0)) return nan("");
    const double logLaw = log(wallDist / z0);
    const double uN = fmax(0.0, (kappa * U) / logLaw);
    if (fabs(qwall) < 1e-6) return uN;
    double u0 = uN, diff;
    int iter = 0;
    do {
        const double L0 = clamp_l(-pow(u0, 3.0) / (kappa * (kG / thetaRef) * qwall));
        double psiM, psiH;
        psi(wallDist / L0, L0 > 0, gammaM, 0.0, psiM, psiH);
        const double uNew = fmax(0.0, (kappa * U) / (logLaw - psiM));
        u0 = kOmega * uNew + (1.0 - kOmega) * u0;
        diff = fabs(uNew - u0);
        iter++;
    } while (diff > kTol && iter < kIterMax);
    if (iter == kIterMax) return uN;
    const double L = clamp_l(-pow(u0, 3.0) / (kappa * (kG / thetaRef) * qwall));
    if (L > 0 && u0 < 1e-2) return stable_bisection(U, wallDist, z0, gammaM, kappa, qwall, thetaRef, uN);
    return u0;
}

// qWallShumann, wallfunctions.c:133-290: the wall heat flux
__device__ __forceinline__ double qwall(double U, double wallDist, double z0, double gammaM, double gammaH, double alphaH,
                                        double thetaRef, double deltaTheta, double kappa)
{
    if (!(wallDist > z0)) return nan("");
    const double lz = log(wallDist / z0);
    const double uN = fmax(0.0, (kappa * U) / lz);
    double qN = (-deltaTheta * uN * kappa) / (alphaH * lz);
    if (fabs(qN) < 1e-6) qN = (qN < 0 ? -1.0 : 1.0) * 1e-6;
    if (deltaTheta == 0.0) return qN;
    double u0 = uN, q0 = qN, du, dq;
    int iter = 0;
    do {
        const double L0 = clamp_l(-pow(u0, 3.0) / (kappa * (kG / thetaRef) * q0));
        double psiM, psiH;
        psi(wallDist / L0, L0 > 0, gammaM, gammaH, psiM, psiH);
        const double uNew = fmax(0.0, (kappa * U) / (lz - psiM));
        u0 = kOmega * uNew + (1.0 - kOmega) * u0;
        const double qNew = (-deltaTheta * u0 * kappa) / (alphaH * lz - psiH);
        q0 = kOmega * qNew + (1.0 - kOmega) * q0;
        du = fabs(uNew - u0);
        dq = fabs(qNew - q0);
        iter++;
    } while ((du > kTol || dq > kTol) && iter < kIterMax);
    if (iter == kIterMax) return qN;
    const double L = clamp_l(-pow(u0, 3.0) / (kappa * (kG / thetaRef) * q0));
    if (L > 0 && u0 < 1e-2) {
        const double us = stable_bisection(U, wallDist, z0, gammaM, kappa, qN, thetaRef, uN);
        const double Lf = fmax(1e-10, -pow(us, 3.0) / (kappa * (kG / thetaRef) * qN));
        const double psiH = -gammaH * (wallDist / Lf);
        return (-deltaTheta * us * kappa) / (alphaH * lz - psiH);
    }
    return q0;
}

}  // namespace mo

}  // namespace tg
