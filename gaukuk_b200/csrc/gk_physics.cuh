// gk_physics.cuh -- pointwise device physics of the finite-volume update.
//
// Included inside the mode namespace (gk_parity / gk_fast).  Every
// expression keeps the reference's association order.  The parity unit is
// compiled with -fmad=false and uses IEEE division and square root, which
// are correctly rounded on the GPU as on the host: results are bit-identical
// to the reference built without -ffast-math.  The fast unit (GK_FASTMATH) lets the
// compiler contract to FMA and replaces division, reciprocal and square root
// by the branch-free refinements below.
#pragma once

// libstdc++ std::max / std::min: max(a,b) = (a<b)?b:a, min(a,b) = (b<a)?b:a.
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }

#if GK_FASTMATH
// Reciprocal, quotient and square root for finite, positive, normal
// arguments (densities, pressures, sound speeds, wave-speed differences).
// Each starts from the hardware approximation (PTX rcp.approx.ftz.f64 /
// rsqrt.approx.ftz.f64, about 2^-22 relative error) and applies one
// third-order step of the binomial series, which cubes the relative error:
//   reciprocal  e = 1 - b*y,    y' = y*(1 + e + e^2)
//   rsqrt       d = 1 - x*y^2,  y' = y*(1 + d/2 + 3d^2/8)
// (the series of (1 - e)^-1 and (1 - d)^-1/2 to second order; one step does
// the work of two Newton steps in fewer operations).  The square root is
// x*rsqrt(x) with one Newton correction of the residual x - s*s (Markstein,
// IBM J. Res. Dev. 34(1), 1990).  The result is within a few ulp of the IEEE
// value; there is no slow path and no branch.
__device__ __forceinline__ double rcp_nr(double b) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    const double e = fma(-b, y, 1.0);
    return fma(y, fma(e, e, e), y);
}
__device__ __forceinline__ double rsqrt_nr(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double d = fma(-x * y, y, 1.0);
    return fma(y, d * fma(0.375, d, 0.5), y);
}
__device__ __forceinline__ double sqrt_nr(double x) {
    const double y = rsqrt_nr(x);
    const double s = x * y;
    const double r = fma(-s, s, x);
    return fma(r, 0.5 * y, s);
}
#define GK_DIV(a, b) ((a) * rcp_nr(b))
#define GK_RCP(b) rcp_nr(b)
#define GK_SQRT(x) sqrt_nr(x)

// Fast mode's sign and order decisions on the integer pipes, from the bit
// patterns: the FP64 pipe bounds the stage kernel, and a compare there costs
// as much as an add.  They differ from the IEEE compares only on -0 and on
// NaNs (fast mode's contract is a tolerance; a non-finite state is still
// caught by the CFL reduction).
__device__ __forceinline__ double pos_part(double x) {  // max(x, 0)
    return __double2hiint(x) < 0 ? 0.0 : x;
}
__device__ __forceinline__ double neg_part(double x) {  // min(0, x)
    return __double2hiint(x) < 0 ? x : 0.0;
}
__device__ __forceinline__ bool ge0(double x) { return __double2hiint(x) >= 0; }        // x >= 0
__device__ __forceinline__ bool le0(double x) { return __double_as_longlong(x) <= 0; }  // x <= 0
// max(x, f) for a positive floor f (signed 64-bit order of the patterns is
// the order of the values when f > 0)
__device__ __forceinline__ double floor_at(double x, double f) {
    return __double_as_longlong(x) < __double_as_longlong(f) ? f : x;
}
#define GK_MAX0(x) pos_part(x)
#define GK_MIN0(x) neg_part(x)
#define GK_GE0(x) ge0(x)
#define GK_LE0(x) le0(x)
#define GK_FLOOR(x, f) floor_at((x), (f))
#define GK_BELOW(x, f) (__double_as_longlong(x) < __double_as_longlong(f))
// max of two non-negative values (speeds): their bit patterns order alike
#define GK_MAXNN(a, b) (__double_as_longlong(a) < __double_as_longlong(b) ? (b) : (a))
#else
// Parity mode: IEEE division and square root (correctly rounded on the GPU
// as on the host).
#define GK_DIV(a, b) ((a) / (b))
#define GK_RCP(b) (1.0 / (b))
#define GK_SQRT(x) sqrt(x)
// the reference's compares and std::max/min
#define GK_MAX0(x) smax((x), 0.0)
#define GK_MIN0(x) smin(0.0, (x))
#define GK_GE0(x) ((x) >= 0)
#define GK_LE0(x) ((x) <= 0.0)
#define GK_FLOOR(x, f) smax((x), (f))
#define GK_BELOW(x, f) ((x) < (f))
#define GK_MAXNN(a, b) smax((a), (b))
#endif

// Reconstruction::VanLeer (reconstruction.hpp:36-42).
__device__ __forceinline__ double vanleer(double a, double b) {
    double multi = a * b;
#if GK_FASTMATH
    double sigma = GK_DIV(2.0 * multi, a + b);
    return (multi <= 0.0) ? 0.0 : sigma;
#else
    return (multi <= 0.0) ? 0.0 : GK_DIV(2.0 * multi, a + b);
#endif
}

#if GK_FASTMATH
// Half the van Leer slope, (a*b)/(a+b) for ab > 0 else 0: what the PLM face
// states u +- 0.5*sigma add, without the two scalings by 2 and 1/2.
__device__ __forceinline__ double vanleer_half(double a, double b) {
    const double multi = a * b;
    const double h = GK_DIV(multi, a + b);
    return GK_LE0(multi) ? 0.0 : h;
}
#endif

struct Flux5 {
    double d, n, t1, t2, e;  // density, normal momentum, tangential 1/2, energy
};

// Flux::RiemannSolver for one face (hllc.cpp:22-101), HLLC after Toro
// ch. 10 with the PVRS pressure estimate.  Velocities come as (normal,
// tangential 1, tangential 2) in the reference's rotation
// (IVLX, IVLY, IVLZ = hllc.cpp:25-27).  T2 = false drops the second
// tangential component, which callers use only when it is exactly zero (2D
// runs with vz = 0): every term it contributes is then an exact zero.
//
// SEL picks how the two star sides are combined, f = selectl*fl + selectr*fr
// with selectl = (ss >= 0) ? 1 : 0 (hllc.cpp:75-94): 0 both sides, as the
// reference writes it (parity mode); 1 only the selected side (fast mode),
// which differs only where the unused side is not finite, or in the sign of
// a zero.
template <bool T2, int SEL>
__device__ __forceinline__ void hllc(double denl, double vxl, double vyl, double vzl, double prel,
                                     double denr, double vxr, double vyr, double vzr, double prer,
                                     const gk::Phys& ph, Flux5& f) {
    const double gamma = ph.gamma;
#if GK_FASTMATH
    // sqrt(gamma*p/rho) = (gamma*p) * rsqrt(gamma*p*rho): one root, no quotient
    const double gpl = gamma * prel, gpr = gamma * prer;
    double al = gpl * rsqrt_nr(gpl * denl);
    double ar = gpr * rsqrt_nr(gpr * denr);
#else
    // EquationOfState::SoundSpeed (eos.hpp:27-29)
    double al = GK_SQRT(GK_DIV(gamma * prel, denl));
    double ar = GK_SQRT(GK_DIV(gamma * prer, denr));
#endif
    double prePVRS = 0.5 * (prel + prer) - 0.125 * (vxr - vxl) * (denl + denr) * (al + ar);
    prePVRS = GK_MAX0(prePVRS);
#if GK_FASTMATH
    // a*q = sqrt(gamma p/rho) * sqrt(1 + cq max(p*/p - 1, 0)) = sqrt(gamma X/rho)
    // with X = p + cq max(p* - p, 0): one root per side, no quotient.
    // Branch-free on purpose: a skip when p* <= p (as in parity mode) was
    // measured slower, because it splits the straight-line code in which the
    // x- and y-face solves of a row interleave.
    const double gxl = fma(ph.gcq, GK_MAX0(prePVRS - prel), gpl);
    const double gxr = fma(ph.gcq, GK_MAX0(prePVRS - prer), gpr);
    // S - v = -+ gX rsqrt(gX rho), so rho (S - v) = -+ (gX rho) rsqrt(gX rho)
    const double xl = gxl * denl, xr = gxr * denr;
    const double rl = rsqrt_nr(xl), rr = rsqrt_nr(xr);
    double sl = vxl - gxl * rl;
    double sr = vxr + gxr * rr;
#else
    double ql, qr;
    // q = sqrt(1 + 0.5*(1+1/gamma)*max(p*/p - 1, 0)) is exactly 1 whenever
    // p* <= p with p > 0, so the division and root are skipped there.
    ql = 1.0;
    qr = 1.0;
    if (!(prePVRS <= prel && prel > 0.0)) {
        double temp = smax(GK_DIV(prePVRS, prel) - 1, 0.0);
        ql = GK_SQRT(1 + ph.cq * temp);
    }
    if (!(prePVRS <= prer && prer > 0.0)) {
        double temp = smax(GK_DIV(prePVRS, prer) - 1, 0.0);
        qr = GK_SQRT(1 + ph.cq * temp);
    }
    double sl = vxl - al * ql;
    double sr = vxr + ar * qr;
#endif
#if GK_FASTMATH
    // the contact speed with rho (S - v) of each side formed once
    const double ml = -(xl * rl), mr = xr * rr;
    double ss = GK_DIV(prer - prel + ml * vxl - mr * vxr, ml - mr);
#else
    double ss = GK_DIV(prer - prel + denl * vxl * (sl - vxl) - denr * vxr * (sr - vxr),
                       denl * (sl - vxl) - denr * (sr - vxr));
#endif
    auto both_sides = [&]() {
        // EquationOfState::EGas (eos.hpp:30-32) + kinetic energy
        double kl = T2 ? (vxl * vxl + vyl * vyl + vzl * vzl) : (vxl * vxl + vyl * vyl);
        double kr = T2 ? (vxr * vxr + vyr * vyr + vzr * vzr) : (vxr * vxr + vyr * vyr);
        double el = prel * ph.gm1Rec + 0.5 * denl * kl;
        double er = prer * ph.gm1Rec + 0.5 * denr * kr;
        double cl = GK_DIV(smin(0.0, sl) * (ss - vxl), sl - ss);
        double cr = GK_DIV(smax(0.0, sr) * (ss - vxr), sr - ss);
        double selectl = (ss >= 0) ? 1.0 : 0.0;
        double selectr = 1.0 - selectl;
        double fl1 = denl * (vxl + cl);
        double fl2 = denl * (vxl * vxl + cl * sl) + prel;
        double fl3 = fl1 * vyl;
        double fl5 = (el + prel) * (vxl + cl) + denl * cl * ss * (sl - vxl);
        double fr1 = denr * (vxr + cr);
        double fr2 = denr * (vxr * vxr + cr * sr) + prer;
        double fr3 = fr1 * vyr;
        double fr5 = (er + prer) * (vxr + cr) + denr * cr * ss * (sr - vxr);
        f.d = selectl * fl1 + selectr * fr1;
        f.n = selectl * fl2 + selectr * fr2;
        f.t1 = selectl * fl3 + selectr * fr3;
        if (T2) {
            double fl4 = fl1 * vzl;
            double fr4 = fr1 * vzr;
            f.t2 = selectl * fl4 + selectr * fr4;
        } else {
            f.t2 = 0.0;
        }
        f.e = selectl * fl5 + selectr * fr5;
    };
    if (SEL == 0) {
        both_sides();
        return;
    }
    // The selected side only (fast mode): its kinetic energy from the
    // selected velocities, and E + p as p/(gamma-1) + p + rho k/2 in one
    // product with gamma/(gamma-1).  m = rho (S - v) of the side, formed for
    // the contact speed, carries the star-state terms:
    //   rho (vn^2 + c S) = f1 vn + c m,   rho c ss (S - vn) = c ss m.
    const bool left = GK_GE0(ss);
    double d = left ? denl : denr, vn = left ? vxl : vxr, v1 = left ? vyl : vyr;
    double v2 = left ? vzl : vzr, p = left ? prel : prer, s = left ? sl : sr;
#if GK_FASTMATH
    const double m = left ? ml : mr;
#else
    const double m = d * (s - vn);  // unused: parity mode evaluates both sides
#endif
    double k = T2 ? (vn * vn + v1 * v1 + v2 * v2) : (vn * vn + v1 * v1);
    double ep = p * ph.gm1Rec1 + 0.5 * d * k;  // E + p
    double sc = left ? GK_MIN0(s) : GK_MAX0(s);
    double c = GK_DIV(sc * (ss - vn), s - ss);
    double vc = vn + c;
    double f1 = d * vc;
    f.d = f1;
    f.n = f1 * vn + (c * m + p);
    f.t1 = f1 * v1;
    f.t2 = T2 ? f1 * v2 : 0.0;
    f.e = ep * vc + c * ss * m;
}
