// ysg_model.cuh -- device layout of the earth model and event constants.
//
// The host (module_model.f90:175-383 restated in host/model.cpp) produces the
// normalised knot values and the per-layer natural-spline second derivatives.
// On the device each knot is one 256-byte record so that a spline evaluation
// on knot interval i touches two adjacent records; the whole table (51 KB at
// 200 knots, 102 KB at 400) is staged into shared memory by a TMA bulk copy.
#pragma once
#include "ysg_cplx.cuh"

namespace ysg {

// Parameter slots of a knot record (module_model.f90:129-160).
enum Param {
    P_RHO = 0, P_ACON, P_CCON, P_FCON, P_LCON, P_NCON, P_KAPPA, P_MU,
    P_QKAPPA, P_QMU, P_GRAV, P_XLAM, P_XA2, NPARAM
};

struct Knot {
    double r, alpha, beta;
    double inv_a2;             // 1 / (alpha alpha), rounded as the start-level search forms it
    double v[NPARAM][2];       // value, spline second derivative
    double inv_b2;             // 1 / (beta beta), the same
    double r2;                 // r r, the same
};
static_assert(sizeof(Knot) == 256, "knot record must be 256 bytes");

// The derived fields of a knot record: the start-level search
// (module_start.f90:14-178) forms 1/v^2 and r^2 of every knot it visits for
// every solve; each is one correctly rounded operation of the knot's own
// values, formed here once per model instead.  A zero speed (a fluid's
// beta) gives +inf, as the search's own quotient does.
inline __host__ __device__ void knot_derive(Knot& k)
{
    k.inv_a2 = 1.0 / (k.alpha * k.alpha);
    k.inv_b2 = 1.0 / (k.beta * k.beta);
    k.r2 = k.r * k.r;
}

// Scalar part of the model.  Indices are 1-based as in the reference.
struct ModelHdr {
    int nknot, nic, noc, nsl, ocean, fic;
    int imin_alpha;      // iminloc(alpha)            (module_int.f90:1157)
    int imin_beta;       // iminloc(beta(noc+1:nsl))+noc (module_int.f90:200-201)
    double tref;         // normalised reference angular frequency
    double pibigg;       // module_model.f90:490
    double fre_norm;     // module_model.f90:484
    double pad;
};

// Per-event constants of the (omega,l) loop (yspec.f90:176-261).
struct EventDev {
    int lmin, lmax, nw, is, ir, ats, grav, out, cor, nr;
    int jofs, jstride;   // frequency shard: local j -> full-band index jofs + (j-1) jstride
    int pot;             // 1: potential coefficients in place of the displacement ones
    double rs, rr, ep, wmin, dw, grav_ir;
    double mm[6];
};

// Number of l-sum coefficients per (omega,l): uu(1:5), vv(1:5), ww(1:5).
constexpr int NCOEF = 15;

// Knot-interval spline evaluator (module_spline.f90:262-283).  The interval
// weights are formed once per radius and reused for every parameter.
struct SplPt {
    double A, B, A3, B3, h26;
    int lo;
    bool flat;
};

__device__ __forceinline__ SplPt spl_at(const Knot* kn, int klo, double x)
{
    SplPt s;
    s.lo = klo;
    double xa = kn[klo].r, xb = kn[klo + 1].r;
    double h = xb - xa;
    s.flat = (h == 0.0);
    double ih = s.flat ? 0.0 : 1.0 / h;
    s.A = (xb - x) * ih;
    s.B = (x - xa) * ih;
    s.A3 = s.A * s.A * s.A - s.A;
    s.B3 = s.B * s.B * s.B - s.B;
    s.h26 = h * h * (1.0 / 6.0);
    return s;
}

__device__ __forceinline__ double spl(const Knot* kn, const SplPt& s, int p)
{
    const Knot& a = kn[s.lo];
    if (s.flat) return a.v[p][0];
    const Knot& b = kn[s.lo + 1];
    return s.A * a.v[p][0] + s.B * b.v[p][0] + (s.A3 * a.v[p][1] + s.B3 * b.v[p][1]) * s.h26;
}

// The same cubic on knot interval i in power form, value = c0 + t (c1 +
// t (c2 + t c3)) with t = r - r_i.  Expanding A y_i + B y_i+1 + ((A^3-A) y''_i
// + (B^3-B) y''_i+1) h^2/6 in t = B h gives
//   c0 = y_i,  c1 = (y_i+1 - y_i)/h - h (2 y''_i + y''_i+1)/6,
//   c2 = y''_i / 2,  c3 = (y''_i+1 - y''_i) / (6 h),
// and c1 = c2 = c3 = 0 on a zero-length interval.  The right-hand sides
// evaluate the model with it: three fused multiply-adds per parameter and
// no division, equal to the form above to rounding.  Record i covers
// [r_i, r_i+1] (1-based like the knots); 432 bytes, 16-byte aligned.
struct __align__(16) Seg {
    double r0, pad;
    double c[NPARAM][4];
};
static_assert(sizeof(Seg) == 432, "segment record size");

// Unit model directions of the reverse sweep, one per parameter: knot
// records with v[p][0] = 1 for parameter p and zero elsewhere, and the
// segments of the same (c[p][0] = 1).
struct UnitDirs {
    const Knot* kn[NPARAM];
    const Seg* sg[NPARAM];
};

__device__ __forceinline__ double seg(const Seg& s, double t, int p)
{
    // two 128-bit loads through the read-only path (the table never changes
    // during a launch)
    const double2* c = reinterpret_cast<const double2*>(s.c[p]);
    const double2 lo = __ldg(c), hi = __ldg(c + 1);
    return fma(fma(fma(hi.y, t, hi.x), t, lo.y), t, lo.x);
}

}  // namespace ysg
