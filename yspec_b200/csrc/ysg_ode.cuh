// ysg_ode.cuh -- per-(omega,l) radial solves on the device.
//
// Device restatement of the reference's ODE machinery:
//   module_int.f90    coefficient matrices, minor / b-vector systems, start
//                     values, minor algebra, Cash-Karp stepping (yint/rkck),
//                     per-solve constants (set_l/set_omega/steps)
//   module_start.f90  start-level search
//   module_solver.f90 the BVP drivers and source vectors
// The reference keeps solve state in module globals; here it is a Ctx in
// registers, so every thread can run an independent (omega,l) solve.
//
// Quantities that steer integer decisions (start level, step counts, grid
// points of the l = 0 gravity solve) are formed with explicitly rounded
// operations so they agree bit for bit with the reference's unfused FP64.
#include "ysg_dual.cuh"
#include "ysg_model.cuh"

// Five builds of the solver code exist: the plain form keeps the Cash-Karp
// stage vectors in per-thread arrays (the compiler places them in local
// memory); with YSG_SMEM_STAGES the stage vectors live in a per-thread slab
// of shared memory and only y and the stage input stay in registers; with
// YSG_COUNT_ONLY yint only counts the steps it would take (the cost model of
// the pair scheduler: every integer decision of a solve -- start levels,
// layers, step counts -- is made as in a real solve, no state is stepped);
// with YSG_TANGENT every quantity that depends on the earth model is a dual
// number (ysg_dual.cuh) and the solve returns, beside its value, the
// derivative along one direction of the model (the tangent-linear solver);
// with YSG_LOOPED_STEP the plain solve takes the looped Cash-Karp step of
// the tangent build (one right-hand side in the code instead of six), for
// kernels whose instruction footprint matters more than the step's
// registers (the reverse sweep).
// Each form gets its own inline namespace so the translation units never
// share a definition, and a translation unit may include this header once
// per form (the reverse sweep uses the plain and the tangent form): the
// include guard is per form.
#ifndef YSG_SMEM_STAGES
#define YSG_SMEM_STAGES 0
#endif
#ifndef YSG_COUNT_ONLY
#define YSG_COUNT_ONLY 0
#endif
#ifndef YSG_TANGENT
#define YSG_TANGENT 0
#endif
#ifndef YSG_LOOPED_STEP
#define YSG_LOOPED_STEP 0
#endif
#undef YSG_VARIANT
#undef YSG_ODE_BODY
#if YSG_TANGENT
#define YSG_VARIANT v_tangent
#ifndef YSG_ODE_DONE_v_tangent
#define YSG_ODE_DONE_v_tangent
#define YSG_ODE_BODY
#endif
#elif YSG_COUNT_ONLY
#define YSG_VARIANT v_count
#ifndef YSG_ODE_DONE_v_count
#define YSG_ODE_DONE_v_count
#define YSG_ODE_BODY
#endif
#elif YSG_SMEM_STAGES
#define YSG_VARIANT v_smem
#ifndef YSG_ODE_DONE_v_smem
#define YSG_ODE_DONE_v_smem
#define YSG_ODE_BODY
#endif
#elif YSG_LOOPED_STEP
#define YSG_VARIANT v_loop
#ifndef YSG_ODE_DONE_v_loop
#define YSG_ODE_DONE_v_loop
#define YSG_ODE_BODY
#endif
#else
#define YSG_VARIANT v_local
#ifndef YSG_ODE_DONE_v_local
#define YSG_ODE_DONE_v_local
#define YSG_ODE_BODY
#endif
#endif
// Helpers on plain and dual complex values only: the same in every form,
// so they sit outside the per-form namespaces (argument-dependent lookup
// on cd would otherwise see one copy per form included).
#ifndef YSG_ODE_COMMON
#define YSG_ODE_COMMON
namespace ysg {

__device__ __forceinline__ double norm2(cd a) { return a.x * a.x + a.y * a.y; }

// Complex multiply-accumulate s + x y (cmac) and s - x y (cmsc) as fused
// multiply-adds: four for a complex factor, two for a real one, where a
// product followed by a sum takes six and four.  The 14-component systems
// accumulate their outputs term by term with them, in the tangent build
// too (the value and the derivative part each fused).
__device__ __forceinline__ cd cmac(cd s, cd x, cd y)
{
    return cd{fma(x.x, y.x, fma(-x.y, y.y, s.x)), fma(x.x, y.y, fma(x.y, y.x, s.y))};
}
__device__ __forceinline__ cd cmsc(cd s, cd x, cd y)
{
    return cd{fma(-x.x, y.x, fma(x.y, y.y, s.x)), fma(-x.x, y.y, fma(-x.y, y.x, s.y))};
}
__device__ __forceinline__ cd cmac(cd s, double x, cd y) { return cd{fma(x, y.x, s.x), fma(x, y.y, s.y)}; }
__device__ __forceinline__ cd cmsc(cd s, double x, cd y) { return cd{fma(-x, y.x, s.x), fma(-x, y.y, s.y)}; }
__device__ __forceinline__ cd cmac(cd s, cd x, double y) { return cmac(s, y, x); }
__device__ __forceinline__ cd cmsc(cd s, cd x, double y) { return cmsc(s, y, x); }
// dual numbers: the value and d(s + x y) = ds + dx y + x dy, both fused
__device__ __forceinline__ dcplx cmac(dcplx s, dcplx x, dcplx y)
{
    return dcplx(cmac(s.v, x.v, y.v), cmac(cmac(s.d, x.d, y.v), x.v, y.d));
}
__device__ __forceinline__ dcplx cmsc(dcplx s, dcplx x, dcplx y)
{
    return dcplx(cmsc(s.v, x.v, y.v), cmsc(cmsc(s.d, x.d, y.v), x.v, y.d));
}
__device__ __forceinline__ dcplx cmac(dcplx s, dreal x, dcplx y)
{
    return dcplx(cmac(s.v, x.v, y.v), cmac(cmac(s.d, x.d, y.v), x.v, y.d));
}
__device__ __forceinline__ dcplx cmsc(dcplx s, dreal x, dcplx y)
{
    return dcplx(cmsc(s.v, x.v, y.v), cmsc(cmsc(s.d, x.d, y.v), x.v, y.d));
}
__device__ __forceinline__ dcplx cmac(dcplx s, dcplx x, dreal y) { return cmac(s, y, x); }
__device__ __forceinline__ dcplx cmsc(dcplx s, dcplx x, dreal y) { return cmsc(s, y, x); }
template <class S, class X, class Y>
__device__ __forceinline__ S cmac(S s, X x, Y y)
{
    return s + x * y;
}
template <class S, class X, class Y>
__device__ __forceinline__ S cmsc(S s, X x, Y y)
{
    return s - x * y;
}

}  // namespace ysg
#endif  // YSG_ODE_COMMON

#ifdef YSG_ODE_BODY

namespace ysg {
inline namespace YSG_VARIANT {

// Types of the quantities that depend on the earth model: model values and
// everything formed from them (coefficient matrices, start vectors, the
// solution).  Plain doubles and complex values except in the tangent build.
// Quantities that depend only on omega, l and the radius stay double / cd.
#if YSG_TANGENT
using mreal = dreal;
using mcplx = dcplx;
#else
using mreal = double;
using mcplx = cd;
#endif

// nrtype.f90:18-27: pi_d and twopi_d are single-precision literals.
constexpr double PI_D = (double)3.14159265358979323846f;
constexpr double TWOPI_D = (double)6.28318530717958647692f;
constexpr double FOURPI_D = 12.56637061;
constexpr double SC_TINY = 1.0e-20;           // module_int.f90:80
constexpr double SC_HUGE = 1.0 / 1.0e-20;     // module_int.f90:81
constexpr int NW_STEP = 4;                    // module_int.f90:74
constexpr double TOL_START = 11.0;            // module_start.f90:6

// Step counters per system (index = Sys::CLS), for the algorithmic work
// model: 0 toroidal, 1 radial, 2 fluid minors ng/cow, 3 b-vector ng/cow,
// 4 solid minors ng/cow, 5 fluid minors g, 6 solid minors g, 7 b-vector g.
constexpr int NSYS = 8;

struct Ctx {
    const Knot* kn;
    const ModelHdr* mh;
    int ll, llp1, il;
    unsigned nst[NSYS];
    const Seg* sg;   // power-form spline segments (right-hand sides)
    cd* kb;          // shared-memory stage slab of this thread (smem form)
#if YSG_COUNT_ONLY
    const int* pfx;  // steps of the whole knot intervals below k, summed, at this omega (or null)
#endif
#if YSG_TANGENT
    const Knot* dkn; // derivative of the knot values along the model direction
    const Seg* dsg;  // derivative of the power-form segments
#endif
    double zeta, zeta2, zeta2m2, szeta2m2, nu, dr, ats;
    double pib;      // pi * bigg of the model (module_model.f90:490), = mh->pibigg
    cd omega, omega2, omegai, omegai2, lno;
};

// module_int.f90:2072-2089
__device__ __forceinline__ void set_l(Ctx& c, int l)
{
    c.ll = l;
    c.llp1 = l + 1;
    c.zeta2 = (double)(float)(l * (l + 1));
    c.zeta = sqrt(c.zeta2);
    c.zeta2m2 = c.zeta2 - 2.0;
    c.szeta2m2 = c.zeta2m2 > 0.0 ? sqrt(c.zeta2m2) : 0.0;
    c.nu = sqrt((double)(float)(2 * l + 1) / FOURPI_D);
}

// module_int.f90:2091-2102
__device__ __forceinline__ void set_omega(Ctx& c, cd w)
{
    c.omega = w;
    c.omega2 = w * w;
    c.omegai = 1.0 / w;
    c.omegai2 = c.omegai * c.omegai;
    if (YSG_COUNT_ONLY) {          // the attenuation term steers no integer decision
        c.lno = mk(0.0);
        return;
    }
    cd z = imul(w) / c.mh->tref;
    c.lno = c.ats * ((2.0 * clog(z)) / PI_D);
}

// module_int.f90:2121-2138
__device__ __forceinline__ double steps(const Ctx& c, int i)
{
    const Knot* kn = c.kn;
    double tmp = i < c.mh->nknot ? fmax(kn[i].alpha, kn[i + 1].alpha) : kn[i].alpha;
    double s = __dmul_rn((double)NW_STEP, c.omega.x) / tmp;
    return 1.0 / s;
}

// module_int.f90:1145-1166 sph_steps / :394-414 rad_steps
__device__ __forceinline__ void alpha_steps(Ctx& c)
{
    double a = c.kn[c.mh->imin_alpha].alpha;
    c.dr = (c.omega.x == 0.0) ? 1.0 / NW_STEP : 1.0 / (__dmul_rn((double)NW_STEP, c.omega.x) / a);
}

// Model value of parameter p on the current layer at offset u from its
// base (power form), and at a knot-interval spline point (start values,
// source vectors); duals in the tangent build.
__device__ __forceinline__ mreal segr(const Ctx& c, const Seg& g, double u, int p)
{
#if YSG_TANGENT
    return mreal(seg(g, u, p), seg(c.dsg[c.il], u, p));
#else
    return seg(g, u, p);
#endif
}

__device__ __forceinline__ mreal splr(const Ctx& c, const SplPt& s, int p)
{
#if YSG_TANGENT
    return mreal(spl(c.kn, s, p), spl(c.dkn, s, p));
#else
    return spl(c.kn, s, p);
#endif
}

// ---------------------------------------------------------------------------
// Coefficient matrices
//
// The model is evaluated from the power-form segments of the current layer
// (c.il, set by yint).  The reference's separate divisions (1/r and the
// complex reciprocals 1/(C(1 + qa lno)), 1/(L(1 + qmu lno))) are formed from
// one real division: for a real c and complex q, 1/(c q) = conj(q) / (c |q|^2),
// and the real denominators are multiplied together and split back out.
// The moduli are O(1) after normalisation, so this stays far from overflow
// and agrees with the separate divisions to a few ulps.
// ---------------------------------------------------------------------------

// module_int.f90:134-164 tor_amat (t real, k and s complex)
struct TorCoef { mreal t; mcplx k, s; };

__device__ __forceinline__ TorCoef tor_amat(const Ctx& c, double rr)
{
    const Seg& g = c.sg[c.il];
    const double u = rr - g.r0;
    mreal rrho = segr(c, g, u, P_RHO), rlcon = segr(c, g, u, P_LCON);
    mreal rncon = segr(c, g, u, P_NCON), rqmu = segr(c, g, u, P_QMU);
    mcplx qll = 1.0 + rqmu * c.lno;
    mcplx cncon = rncon * qll;
    const mreal dl = rlcon * norm2(qll);
    const mreal inv = 1.0 / (rr * dl);
    mreal ri = dl * inv;
    TorCoef a;
    a.t = 2.0 * ri;
    a.k = conj(qll) * (rr * inv);     // 1 / (L (1 + qmu lno))
    a.s = -(c.omega2 * rrho) + (ri * ri * c.zeta2m2) * cncon;
    return a;
}

// module_int.f90:261-304 rad_amat.  rad_derivs_ng also calls this gravity
// form (module_int.f90:388), so both radial systems share it.
struct RadCoef { mcplx t, k, s; };

__device__ __forceinline__ RadCoef rad_amat(const Ctx& c, double rr)
{
    const Seg& g = c.sg[c.il];
    const double u = rr - g.r0;
    mreal rrho = segr(c, g, u, P_RHO), racon = segr(c, g, u, P_ACON), rccon = segr(c, g, u, P_CCON);
    mreal rfcon = segr(c, g, u, P_FCON), rncon = segr(c, g, u, P_NCON), gg = segr(c, g, u, P_GRAV);
    mreal rqmu = segr(c, g, u, P_QMU), rxlam = segr(c, g, u, P_XLAM), rxa2 = segr(c, g, u, P_XA2);
    mcplx qaa = 1.0 + rxa2 * c.lno, qff = 1.0 + rxlam * c.lno, qll = 1.0 + rqmu * c.lno;
    mcplx cacon = racon * qaa, cfcon = rfcon * qff, cncon = rncon * qll;
    const mreal dc = rccon * norm2(qaa);
    const mreal inv = 1.0 / (rr * dc);
    mcplx cccon = conj(qaa) * (rr * inv);     // 1 / (C (1 + qa lno))
    mcplx gamma = cmsc(cacon - cncon, cfcon * cfcon, cccon);
    mreal ri = dc * inv;
    RadCoef a;
    a.t = (1.0 - 2.0 * cfcon * cccon) * ri;
    a.k = cccon;
    a.s = -(c.omega2 * rrho) + (4.0 * (gamma - rrho * gg * rr)) * (ri * ri);
    return a;
}

// Spheroidal coefficients.  KIND: 2 = self-gravitation
// (module_int.f90:500-560 / 676-715), 1 = Cowling (:619-672 / :751-786),
// 0 = no gravity (:564-616 / :720-747).  Entries that are real in value
// are kept real.
struct SolidCoef {
    mcplx t11, t12, k11, k22, s11, s12, s22;
    mreal t21, t22, t31, t33, k33, s13, s23;
};

template <int KIND>
__device__ __forceinline__ SolidCoef solid_amat(const Ctx& c, double rr)
{
    const Seg& g = c.sg[c.il];
    const double u = rr - g.r0;
    mreal rrho = segr(c, g, u, P_RHO), racon = segr(c, g, u, P_ACON), rccon = segr(c, g, u, P_CCON);
    mreal rfcon = segr(c, g, u, P_FCON), rncon = segr(c, g, u, P_NCON), rlcon = segr(c, g, u, P_LCON);
    mreal rqmu = segr(c, g, u, P_QMU), rxlam = segr(c, g, u, P_XLAM), rxa2 = segr(c, g, u, P_XA2);
    mcplx qaa = 1.0 + rxa2 * c.lno, qff = 1.0 + rxlam * c.lno, qll = 1.0 + rqmu * c.lno;
    mcplx cacon = racon * qaa, cfcon = rfcon * qff, cncon = rncon * qll;
    const mreal dc = rccon * norm2(qaa), dl = rlcon * norm2(qll);
    const mreal inv = 1.0 / (rr * (dc * dl));
    mcplx cccon = conj(qaa) * ((rr * dl) * inv);     // 1 / (C (1 + qa lno))
    mcplx fc = cfcon * cccon;
    mcplx gamma = cmsc(cacon - cncon, cfcon, fc);
    mreal ri = (dc * dl) * inv, ri2 = ri * ri;
    SolidCoef a;
    a.t11 = (1.0 - 2.0 * fc) * ri;
    a.t12 = (c.zeta * ri) * fc;
    a.t21 = -(c.zeta * ri);
    a.t22 = 2.0 * ri;
    a.k11 = cccon;
    a.k22 = conj(qll) * ((rr * dc) * inv);       // 1 / (L (1 + qmu lno))
    mcplx mw2r = -(c.omega2 * rrho);
    a.s22 = mw2r + (c.zeta2 * (gamma + cncon) - 2.0 * cncon) * ri2;
    if (KIND == 0) {
        a.s11 = mw2r + (4.0 * gamma) * ri2;
        a.s12 = (-2.0 * c.zeta) * gamma * ri2;
    } else {
        mreal gg = segr(c, g, u, P_GRAV);
        mreal rgr = rrho * gg * rr;
        a.s11 = mw2r + (4.0 * (gamma - rgr)) * ri2;
        a.s12 = (c.zeta * (rgr - 2.0 * gamma)) * ri2;
    }
    if (KIND == 2) {
        double pib = c.pib;
        a.t31 = -(4.0 * pib * rrho);
        a.t33 = -((double)c.ll * ri);
        a.k33 = 4.0 * pib;
        a.s13 = -(rrho * (double)c.llp1 * ri);
        a.s23 = rrho * c.zeta * ri;
    } else {
        a.t31 = a.t33 = a.k33 = a.s13 = a.s23 = 0.0;
    }
    return a;
}

struct FluidCoef {
    mcplx t11, t12, k11, s11, s12, s22;
    mreal t21, t22, k22;
};

template <int KIND>
__device__ __forceinline__ FluidCoef fluid_amat(const Ctx& c, double rr)
{
    const Seg& g = c.sg[c.il];
    const double u = rr - g.r0;
    mreal rrho = segr(c, g, u, P_RHO), rccon = segr(c, g, u, P_CCON), rxa2 = segr(c, g, u, P_XA2);
    mcplx qaa = 1.0 + rxa2 * c.lno;
    const mreal dc = rccon * norm2(qaa);
    const mreal inv = 1.0 / (rr * rrho * dc);
    mcplx cccon = conj(qaa) * ((rr * rrho) * inv);  // 1 / (C (1 + qa lno))
    mreal ri = (rrho * dc) * inv;
    const mreal irho = (rr * dc) * inv;          // 1 / rho
    FluidCoef a;
    a.k11 = cccon - (c.zeta2 * c.omegai2) * ((ri * ri) * irho);
    if (KIND == 0) {
        a.t11 = mk(-ri);
        a.s11 = -(c.omega2 * rrho);
        a.t12 = a.s12 = a.s22 = mk(0.0);
        a.t21 = a.t22 = a.k22 = 0.0;
        return a;
    }
    mreal gg = segr(c, g, u, P_GRAV);
    mcplx gzw = (gg * c.zeta2) * c.omegai2;
    a.t11 = (gzw * ri - 1.0) * ri;
    a.s11 = -(c.omega2 * rrho) + (rrho * gg) * ((gzw * ri - 4.0) * ri);
    if (KIND == 2) {
        double pib = c.pib;
        a.t12 = (c.zeta2 * c.omegai2) * (ri * ri);
        a.t21 = -4.0 * pib * rrho;
        a.t22 = -((double)c.ll * ri);
        a.k22 = 4.0 * pib;
        a.s12 = rrho * ((gzw * ri - (double)c.llp1) * ri);
        a.s22 = (rrho * c.zeta2 * ri * ri) * c.omegai2;
    } else {
        a.t12 = a.s12 = a.s22 = mk(0.0);
        a.t21 = a.t22 = a.k22 = 0.0;
    }
    return a;
}

// ---------------------------------------------------------------------------
// Right-hand sides.  Each system is a tag type with N components and f().
// ---------------------------------------------------------------------------
struct TorSys {
    static constexpr int N = 2, CLS = 0;
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* y, Out d)
    {
        TorCoef a = tor_amat(c, r);       // module_int.f90:168-184
        d[0] = cmac(a.t * y[0], a.k, y[1]);
        d[1] = cmsc(a.s * y[0], a.t, y[1]);
    }
};

struct RadSys {
    static constexpr int N = 2, CLS = 1;
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* y, Out d)
    {
        RadCoef a = rad_amat(c, r);       // module_int.f90:357-392
        d[0] = cmac(a.t * y[0], a.k, y[1]);
        d[1] = cmsc(a.s * y[0], a.t, y[1]);
    }
};

// module_int.f90:818-871 sph_minors_solid_derivs
struct MinorSolidG {
    static constexpr int N = 14, CLS = 6;
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* m, Out d)
    {
        SolidCoef a = solid_amat<2>(c, r);
        mcplx a123 = a.t11 + (a.t22 + a.t33), a126 = a.t11 + (a.t22 - a.t33);
        mcplx a135 = a.t11 - (a.t22 - a.t33), a234 = (a.t22 + a.t33) - a.t11;
        d[0] = cmac(cmac(cmsc(a.k33 * m[3], a.k22, m[5]), a.k11, m[9]), m[0], a123);
        d[1] = cmsc(cmac(cmsc(cmac(-(a.k22 * m[6]), m[0], a.s13), m[2], a.t21), m[1], a.t22), m[3], a.t31);
        d[2] = cmsc(cmac(cmac(-(a.k11 * m[10]), m[0], a.s23), m[2], a.t11), m[1], a.t12);
        d[3] = cmac(cmsc(a.k22 * m[8], a.k11, m[11]), m[3], a126);
        d[4] = cmac(cmac(cmsc(cmac(cmsc(-(a.k33 * m[7]), m[0], a.s12), m[9], a.t12), m[5], a.t21), m[2], a.t31), m[4], a.t33);
        d[5] = cmac(cmsc(cmsc(cmsc(-(a.k33 * m[8]), a.k11, m[12]), m[0], a.s22), (2.0 * m[4]), a.t12), m[5], a135);
        d[6] = cmac(cmsc(cmac(cmsc(cmsc(cmac(m[2] * a.s12, m[5], a.s13), m[1], a.s22), m[4], a.s23), m[10], a.t12), m[6], a.t22), m[8], a.t31);
        d[7] = cmsc(cmsc(cmac(cmsc(cmsc(m[3] * a.s12, m[2], a.s13), m[1], a.s23), m[11], a.t12), m[8], a.t21), m[7], a.t33);
        d[8] = cmsc(cmsc(cmsc(cmac(a.k11 * m[13], m[3], a.s22), (2.0 * m[2]), a.s23), (2.0 * m[7]), a.t12), m[8], a234);
        d[9] = cmac(cmsc(cmac(cmac(cmac(-(a.k33 * m[11]), a.k22, m[12]), m[0], a.s11), (2.0 * m[4]), a.t21), (2.0 * m[1]), a.t31), m[9], a234);
        d[10] = cmsc(cmac(cmsc(cmsc(cmsc(cmac(-(m[2] * a.s11), m[1], a.s12), m[4], a.s13), m[9], a.s23), m[10], a.t11), m[6], a.t21), m[7], a.t31);
        d[11] = cmsc(cmac(cmac(cmsc(-(a.k22 * m[13]), m[3], a.s11), (2.0 * m[1]), a.s13), (2.0 * m[7]), a.t21), m[11], a135);
        d[12] = cmsc(cmac(cmac(cmac(cmsc(a.k33 * m[13], m[5], a.s11), (2.0 * m[4]), a.s12), m[9], a.s22), (2.0 * m[6]), a.t31), m[12], a126);
        d[13] = cmsc(cmac(cmsc(cmac(cmsc(m[8] * a.s11, (2.0 * m[7]), a.s12), (2.0 * m[6]), a.s13), m[11], a.s22), (2.0 * m[10]), a.s23), m[13], a123);
    }
};

// module_int.f90:874-936 sph_minors_solid_derivs_ng / _cow
template <int KIND>
struct MinorSolidNC {
    static constexpr int N = 5, CLS = 4;
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* m, Out d)
    {
        SolidCoef a = solid_amat<KIND>(c, r);
        mcplx a11 = a.t11 + a.t22, a22 = a.t11 - a.t22;
        d[0] = cmsc(cmac(a11 * m[0], a.k22, m[2]), a.k11, m[3]);
        d[1] = cmac(cmsc(a.s12 * m[0], a.t21, m[2]), a.t12, m[3]);
        d[2] = cmac(cmac(cmsc(a.s22 * m[0], (2.0 * a.t12), m[1]), a22, m[2]), a.k11, m[4]);
        d[3] = cmsc(cmsc(cmac(-(a.s11 * m[0]), (2.0 * a.t21), m[1]), a22, m[3]), a.k22, m[4]);
        d[4] = cmsc(cmsc(cmac(-((2.0 * a.s12) * m[1]), a.s11, m[2]), a.s22, m[3]), a11, m[4]);
    }
};

// module_int.f90:941-967 sph_minors_fluid_derivs
struct MinorFluidG {
    static constexpr int N = 5, CLS = 5;
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* m, Out d)
    {
        FluidCoef a = fluid_amat<2>(c, r);
        mcplx tp = a.t11 + a.t22, tm = a.t11 - a.t22;
        d[0] = cmac(cmsc(a.k22 * m[2], a.k11, m[3]), m[0], tp);
        d[1] = cmsc(cmac(m[0] * a.s12, m[3], a.t12), m[2], a.t21);
        d[2] = cmac(cmsc(cmac(a.k11 * m[4], m[0], a.s22), (2.0 * m[1]), a.t12), m[2], tm);
        d[3] = cmsc(cmac(cmsc(-(a.k22 * m[4]), m[0], a.s11), (2.0 * a.t21), m[1]), m[3], tm);
        d[4] = cmsc(cmsc(cmsc(m[2] * a.s11, (2.0 * m[1]), a.s12), m[3], a.s22), m[4], tp);
    }
};

// module_int.f90:971-1012 sph_minors_fluid_derivs_ng / _cow
template <int KIND>
struct MinorFluidNC {
    static constexpr int N = 2, CLS = 2;
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* m, Out d)
    {
        FluidCoef a = fluid_amat<KIND>(c, r);
        d[0] = cmac(a.t11 * m[0], a.k11, m[1]);
        d[1] = cmsc(a.s11 * m[0], a.t11, m[1]);
    }
};

// module_int.f90:1016-1057 sph_bvec_solid_derivs
struct BvecSolidG {
    static constexpr int N = 14, CLS = 7;
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* b, Out d)
    {
        SolidCoef a = solid_amat<2>(c, r);
        const mcplx t11 = a.t11, t12 = a.t12, k11 = a.k11, k22 = a.k22;
        const mcplx s11 = a.s11, s12 = a.s12, s22 = a.s22;
        const mreal t21 = a.t21, t22 = a.t22, t31 = a.t31, t33 = a.t33, k33 = a.k33;
        const mreal s13 = a.s13, s23 = a.s23;
        d[0] = cmac(cmsc(cmsc(cmsc(cmac(cmac(s11 * b[6], s12, (b[7] - b[2])), s13, b[8]), s22, b[3]), s23, b[4]), (t11 + t22), b[0]), t31, b[5]);
        d[1] = cmsc(cmsc(cmsc(cmsc(cmac(s11 * b[9], s12, b[10]), s13, (2.0 * b[2] + b[7])), s23, b[3]), t21, b[5]), (t11 + t33), b[1]);
        d[2] = cmsc(cmsc(cmac(cmac(s12 * b[11], s13, b[12]), t12, b[3]), t21, b[6]), t31, b[9]);
        d[3] = cmsc(cmac(cmac(cmac(cmsc(-(k22 * b[0]), s11, b[11]), s13, b[13]), t21, (b[2] - b[7])), (t22 - t11), b[3]), t31, b[10]);
        d[4] = cmac(cmac(cmsc(cmsc(cmsc(-(k33 * b[1]), s11, b[12]), s12, b[13]), t21, b[8]), t31, (2.0 * b[2] + b[7])), (t33 - t11), b[4]);
        d[5] = cmsc(cmsc(cmsc(cmac(cmsc(s12 * b[9], s13, b[6]), s22, b[10]), s23, (b[2] + 2.0 * b[7])), t12, b[1]), (t22 + t33), b[5]);
        d[6] = cmac(cmsc(cmac(cmac(k11 * b[0], s22, b[11]), s23, b[12]), t12, (b[2] - b[7])), (t11 - t22), b[6]);
        d[7] = cmac(cmsc(cmac(-(s12 * b[11]), s23, b[13]), t12, b[3]), t21, b[6]);
        d[8] = cmac(cmac(cmsc(cmsc(cmsc(cmsc(-(k33 * b[5]), s12, b[12]), s22, b[13]), t12, b[4]), t22, b[8]), t31, b[6]), t33, b[8]);
        d[9] = cmac(cmac(cmac(k11 * b[1], s23, b[11]), t12, b[10]), (t11 - t33), b[9]);
        d[10] = cmac(cmac(cmsc(k22 * b[5], s13, b[11]), t21, b[9]), (t22 - t33), b[10]);
        d[11] = cmac(cmac(-(k11 * b[3]), k22, b[6]), (t11 + t22), b[11]);
        d[12] = cmac(cmac(cmac(-(k11 * b[4]), k33, b[9]), t12, b[13]), (t11 + t33), b[12]);
        d[13] = cmac(cmsc(cmac(cmac(-(k22 * b[8]), k33, b[10]), t21, b[12]), t31, b[11]), (t22 + t33), b[13]);
    }
};

// The transpose of BvecSolidG's system: d = A^T k for the coefficient
// matrix A of sph_bvec_solid_derivs (module_int.f90:1016-1057).  The
// b-vector solves of the batched form integrate it backwards to obtain only
// the response rows a pair needs (sph_solver_g).
struct BvecSolidGTr {
    static constexpr int N = 14, CLS = 7;
    template <class Out>
    __device__ static __forceinline__ void tr(const SolidCoef& a, const mcplx* k, Out d)
    {
        const mcplx t11 = a.t11, t12 = a.t12, k11 = a.k11, k22 = a.k22;
        const mcplx s11 = a.s11, s12 = a.s12, s22 = a.s22;
        const mreal t21 = a.t21, t22 = a.t22, t31 = a.t31, t33 = a.t33, k33 = a.k33;
        const mreal s13 = a.s13, s23 = a.s23;
        d[0] = cmsc(cmsc(k11 * k[6], (t11 + t22), k[0]), k22, k[3]);
        d[1] = cmsc(cmsc(cmsc(k11 * k[9], (t11 + t33), k[1]), k33, k[4]), t12, k[5]);
        d[2] = cmsc(cmsc(cmsc(cmsc(cmac(t21 * k[3], t31, (2.0 * k[4])), s12, k[0]), s23, k[5]), t12, k[6]), s13, (2.0 * k[1]));
        d[3] = cmsc(cmsc(cmsc(cmsc(cmac(t12 * k[2], (t22 - t11), k[3]), s22, k[0]), s23, k[1]), t12, k[7]), k11, k[11]);
        d[4] = cmsc(cmsc(cmsc((t33 - t11) * k[4], s23, k[0]), t12, k[8]), k11, k[12]);
        d[5] = cmsc(cmsc(cmsc(cmac(t31 * k[0], k22, k[10]), t21, k[1]), (t22 + t33), k[5]), k33, k[8]);
        d[6] = cmsc(cmsc(cmac(cmac(cmac(cmac(s11 * k[0], (t11 - t22), k[6]), t21, k[7]), t31, k[8]), k22, k[11]), t21, k[2]), s13, k[5]);
        d[7] = cmsc(cmsc(cmsc(cmac(cmac(s12 * k[0], t31, k[4]), t12, k[6]), s13, k[1]), t21, k[3]), s23, (2.0 * k[5]));
        d[8] = cmsc(cmsc(cmac(s13 * k[0], (t33 - t22), k[8]), t21, k[4]), k22, k[13]);
        d[9] = cmsc(cmac(cmac(cmac(cmac(s11 * k[1], s12, k[5]), (t11 - t33), k[9]), t21, k[10]), k33, k[12]), t31, k[2]);
        d[10] = cmsc(cmac(cmac(cmac(cmac(s12 * k[1], s22, k[5]), t12, k[9]), (t22 - t33), k[10]), k33, k[13]), t31, k[3]);
        d[11] = cmsc(cmsc(cmsc(cmsc(cmac(cmac(cmac(s12 * k[2], s22, k[6]), s23, k[9]), (t11 + t22), k[11]), s11, k[3]), s12, k[7]), s13, k[10]), t31, k[13]);
        d[12] = cmsc(cmsc(cmac(cmac(cmac(s13 * k[2], s23, k[6]), (t11 + t33), k[12]), t21, k[13]), s11, k[4]), s12, k[8]);
        d[13] = cmsc(cmsc(cmac(cmac(cmac(s13 * k[3], s23, k[7]), t12, k[12]), (t22 + t33), k[13]), s12, k[4]), s22, k[8]);
    }
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* k, Out d)
    {
        tr(solid_amat<2>(c, r), k, d);
    }
};

// module_int.f90:1060-1110 sph_bvec_solid_derivs_ng / _cow
template <int KIND>
struct BvecSolidNC {
    static constexpr int N = 4, CLS = 3;
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* b, Out d)
    {
        SolidCoef a = solid_amat<KIND>(c, r);
        d[0] = cmsc(cmsc(cmsc(-(a.s11 * b[2]), a.s12, b[3]), a.t11, b[0]), a.t21, b[1]);
        d[1] = cmsc(cmsc(cmsc(-(a.s12 * b[2]), a.s22, b[3]), a.t12, b[0]), a.t22, b[1]);
        d[2] = cmac(cmac(-(a.k11 * b[0]), a.t11, b[2]), a.t12, b[3]);
        d[3] = cmac(cmac(-(a.k22 * b[1]), a.t21, b[2]), a.t22, b[3]);
    }
};

// The transpose of BvecSolidNC's system (module_int.f90:1060-1110), for
// the backward response-row integrations of sph_solver_nc.
template <int KIND>
struct BvecSolidNCTr {
    static constexpr int N = 4, CLS = 3;
    template <class Out>
    __device__ static __forceinline__ void f(const Ctx& c, double r, const mcplx* k, Out d)
    {
        const SolidCoef a = solid_amat<KIND>(c, r);
        d[0] = cmsc(cmsc(-(a.t11 * k[0]), a.t12, k[1]), a.k11, k[2]);
        d[1] = cmsc(cmsc(-(a.t21 * k[0]), a.t22, k[1]), a.k22, k[3]);
        d[2] = cmsc(cmsc(cmac(a.t11 * k[2], a.t21, k[3]), a.s11, k[0]), a.s12, k[1]);
        d[3] = cmsc(cmsc(cmac(a.t12 * k[2], a.t22, k[3]), a.s12, k[0]), a.s22, k[1]);
    }
};

// ---------------------------------------------------------------------------
// Cash-Karp RK5 (module_int.f90:2016-2064), fifth-order solution only, with
// the 1e+-20 rescaling of yint (module_int.f90:1910-1919).
// ---------------------------------------------------------------------------
template <class Sys>
__device__ __forceinline__ void rkck_step(const Ctx& c, mcplx* y, double x, double h)
{
    constexpr int N = Sys::N;
    constexpr double a2 = 0.2, a3 = 0.3, a4 = 0.6, a5 = 1.0, a6 = 0.875;
    constexpr double b21 = 0.2, b31 = 3.0 / 40.0, b32 = 9.0 / 40.0;
    constexpr double b41 = 0.3, b42 = -0.9, b43 = 1.2;
    constexpr double b51 = -11.0 / 54.0, b52 = 2.5, b53 = -70.0 / 27.0, b54 = 35.0 / 27.0;
    constexpr double b61 = 1631.0 / 55296.0, b62 = 175.0 / 512.0, b63 = 575.0 / 13824.0,
                     b64 = 44275.0 / 110592.0, b65 = 253.0 / 4096.0;
    constexpr double c1 = 37.0 / 378.0, c3 = 250.0 / 621.0, c4 = 125.0 / 594.0,
                     c6 = 512.0 / 1771.0;
    mcplx k1[N], k2[N], k3[N], k4[N], k5[N], yt[N];
    Sys::f(c, x, y, k1);
    const double hb21 = b21 * h;
#pragma unroll
    for (int i = 0; i < N; i++) yt[i] = y[i] + hb21 * k1[i];
    Sys::f(c, x + a2 * h, yt, k2);
#pragma unroll
    for (int i = 0; i < N; i++) yt[i] = y[i] + h * (b31 * k1[i] + b32 * k2[i]);
    Sys::f(c, x + a3 * h, yt, k3);
#pragma unroll
    for (int i = 0; i < N; i++) yt[i] = y[i] + h * (b41 * k1[i] + b42 * k2[i] + b43 * k3[i]);
    Sys::f(c, x + a4 * h, yt, k4);
#pragma unroll
    for (int i = 0; i < N; i++)
        yt[i] = y[i] + h * (b51 * k1[i] + b52 * k2[i] + b53 * k3[i] + b54 * k4[i]);
    Sys::f(c, x + a5 * h, yt, k5);
#pragma unroll
    for (int i = 0; i < N; i++)
        yt[i] = y[i] + h * (b61 * k1[i] + b62 * k2[i] + b63 * k3[i] + b64 * k4[i] + b65 * k5[i]);
    Sys::f(c, x + a6 * h, yt, k2);   // k6 reuses k2's storage
#pragma unroll
    for (int i = 0; i < N; i++)
        y[i] = y[i] + h * (c1 * k1[i] + c3 * k3[i] + c4 * k4[i] + c6 * k2[i]);
}

// Shared-memory form of the same step: stage vectors go to the thread's
// slab as the right-hand side produces them, so only y and the stage input
// are held in registers.  A warp's slabs are interleaved lane by lane: entry
// e of a lane sits at kb[e * KS], so a warp touches 32 consecutive complex
// values per entry (no bank conflicts) and every offset is a constant.
constexpr int KS = 32;

// Cash-Karp tableau (module_int.f90:2039-2049) for the looped step with
// four slab slots A0..A3.  Stages 1-4 store k1..k4 in A0..A3.  Forming the
// stage-5 input also folds A1 (k2, not needed again: c2 = 0) into the
// partial stage-6 input P6 = b61 k1 + b62 k2 + b63 k3 + b64 k4, and k5 is
// added into it (A1 += b65 k5) as the right-hand side produces it; forming
// the stage-6 input from A1 then folds A1 into the partial increment
// F = c1 k1 + c3 k3 + c4 k4 (c5 = 0), and k6 is added into it
// (A1 += c6 k6); finally y += h A1.  The same sums as the textbook form,
// associated differently.
//   ck_in[s][t]   weight of slot t in the stage-s input (times h)
//   ck_fold[s][t] weight of slot t in the new A1 (stages 5 and 6)
//   ck_slot[s], ck_w[s]: where stage s's derivative goes and with what
//   weight (store for stages 1-4, add for 5 and 6)
__constant__ double ck_a[6] = {0.0, 0.2, 0.3, 0.6, 1.0, 0.875};
__constant__ double ck_in[6][4] = {
    {0.0, 0.0, 0.0, 0.0},
    {0.2, 0.0, 0.0, 0.0},
    {3.0 / 40.0, 9.0 / 40.0, 0.0, 0.0},
    {0.3, -0.9, 1.2, 0.0},
    {-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0},
    {0.0, 1.0, 0.0, 0.0}};
__constant__ double ck_fold[6][4] = {
    {0.0, 0.0, 0.0, 0.0},
    {0.0, 0.0, 0.0, 0.0},
    {0.0, 0.0, 0.0, 0.0},
    {0.0, 0.0, 0.0, 0.0},
    {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0},
    {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0}};
__constant__ int ck_slot[6] = {0, 1, 2, 3, 1, 1};
__constant__ double ck_w[6] = {1.0, 1.0, 1.0, 1.0, 253.0 / 4096.0, 512.0 / 1771.0};

// The step as a runtime loop over the six stages with one copy of the
// right-hand side (six inlined 14-component bodies overflow the
// instruction cache); the stage inputs and the two folds are loops over
// the slots with weights from the tables above, so the step body stays
// small.  Four slots of 14 complex values let four 64-thread blocks share
// an SM.
template <class Sys>
__device__ __forceinline__ void rkck_step_loop(const Ctx& c, cd* y, double x, double h)
{
    constexpr int N = Sys::N;
    constexpr int S = N * KS;                // slot stride in the slab
    cd* const kb = c.kb;
    cd yt[N];
#pragma unroll 1
    for (int s = 0; s < 6; s++) {
#pragma unroll
        for (int i = 0; i < N; i++) yt[i] = y[i];
#pragma unroll 1
        for (int t = 0; t < 4; t++) {
            const double wt = ck_in[s][t];
            if (wt == 0.0) continue;
            const double hb = h * wt;
            const cd* kt = kb + t * S;
#pragma unroll
            for (int i = 0; i < N; i++) yt[i] += hb * kt[i * KS];
        }
        if (s >= 4) {
            const double f0 = ck_fold[s][0], f1 = ck_fold[s][1], f2 = ck_fold[s][2],
                         f3 = ck_fold[s][3];
            cd* const a1 = kb + S;
#pragma unroll 2
            for (int i = 0; i < N; i++) {
                const int o = i * KS;
                a1[o] = f0 * kb[o] + f1 * a1[o] + f2 * kb[2 * S + o] + f3 * kb[3 * S + o];
            }
        }
        // the derivative is formed in registers and written in one pass:
        // stored into its slot (stages 1-4) or added with its weight into A1
        cd d[N];
        Sys::f(c, x + ck_a[s] * h, yt, d);
        if (s < 4) {
            cd* const o = kb + s * S;
#pragma unroll
            for (int i = 0; i < N; i++) o[i * KS] = d[i];
        } else {
            const double w = ck_w[s];
            cd* const o = kb + S;
#pragma unroll
            for (int i = 0; i < N; i++) o[i * KS] += w * d[i];
        }
    }
    const cd* a1 = kb + S;
#pragma unroll
    for (int i = 0; i < N; i++) y[i] = y[i] + h * a1[i * KS];
}

// Transposed step for a linear system y' = A(r) y: w <- M^T w, where M is
// the matrix of one Cash-Karp step at (x, h) (M y = the step's result from
// y).  With Y_s the stage inputs and k_s = A_s Y_s, the step is
// y' = y + h sum_s c_s k_s, Y_s = y + h sum_{t<s} b_st k_t; its transpose
// visits the stages backwards:
//   K_s = h (c_s w + sum_{u>s} b_us G_u),  G_s = A_s^T K_s,
//   w' = w + sum_s G_s.
// The linear system needs no forward state: A_s is formed again at the
// stage radius.  Four slots as in the forward step: G6..G3 are stored in
// A0..A3; forming K2 folds them into A1 = b61 G6 + b51 G5 + b41 G4 + b31 G3
// (the part of K1 still to come) and A0 = G6 + G5 + G4 + G3 (the part of
// w'), G2 is added into both (b21 into A1), K1 = h (c1 w + A1), G1 is added
// into A0, and w' = w + A0.
//   ckt_w[s]      weight of w in K_s (times h)
//   ckt_in[s][t]  weight of slot t in K_s (times h)
__constant__ double ckt_w[6] = {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0};
__constant__ double ckt_in[6][4] = {
    {0.0, 1.0, 0.0, 0.0},
    {175.0 / 512.0, 2.5, -0.9, 9.0 / 40.0},
    {575.0 / 13824.0, -70.0 / 27.0, 1.2, 0.0},
    {44275.0 / 110592.0, 35.0 / 27.0, 0.0, 0.0},
    {253.0 / 4096.0, 0.0, 0.0, 0.0},
    {0.0, 0.0, 0.0, 0.0}};

template <class Sys>
__device__ __forceinline__ void rkck_step_loop_T(const Ctx& c, cd* w, double x, double h)
{
    constexpr int N = Sys::N;
    constexpr int S = N * KS;
    cd* const kb = c.kb;
    cd yt[N];
#pragma unroll 1
    for (int s = 5; s >= 0; s--) {
        const double hw = h * ckt_w[s];
#pragma unroll
        for (int i = 0; i < N; i++) yt[i] = hw * w[i];
#pragma unroll 1
        for (int t = 0; t < 4; t++) {
            const double wt = ckt_in[s][t];
            if (wt == 0.0) continue;
            const double hb = h * wt;
            const cd* kt = kb + t * S;
#pragma unroll
            for (int i = 0; i < N; i++) yt[i] += hb * kt[i * KS];
        }
        if (s == 1) {
            cd* const a1 = kb + S;
#pragma unroll 2
            for (int i = 0; i < N; i++) {
                const int o = i * KS;
                const cd g6 = kb[o], g5 = a1[o], g4 = kb[2 * S + o], g3 = kb[3 * S + o];
                a1[o] = (1631.0 / 55296.0) * g6 + (-11.0 / 54.0) * g5 + 0.3 * g4 + (3.0 / 40.0) * g3;
                kb[o] = (g6 + g5) + (g4 + g3);
            }
        }
        cd d[N];
        Sys::f(c, x + ck_a[s] * h, yt, d);
        if (s >= 2) {
            cd* const o = kb + (5 - s) * S;
#pragma unroll
            for (int i = 0; i < N; i++) o[i * KS] = d[i];
        } else {
#pragma unroll
            for (int i = 0; i < N; i++) kb[i * KS] += d[i];
            if (s == 1) {
#pragma unroll
                for (int i = 0; i < N; i++) kb[S + i * KS] += 0.2 * d[i];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < N; i++) w[i] = w[i] + kb[i * KS];
}

// The looped step with the four slots in a per-thread array (local
// memory) instead of the shared slab, for the tangent build: its dual stage
// vectors are twice the size, and six inlined dual right-hand sides would
// overflow the instruction cache just as the unrolled primal step does.
template <class T>
struct LocalOut {
    T* p;
    double w;
    bool add;
    struct Ref {
        T* a;
        double w;
        bool add;
        __device__ __forceinline__ void operator=(T v) const
        {
            if (add) *a += w * v;
            else *a = v;
        }
    };
    __device__ __forceinline__ Ref operator[](int i) const { return Ref{p + i, w, add}; }
};

template <class Sys>
__device__ __forceinline__ void rkck_step_loop_local(const Ctx& c, mcplx* y, double x, double h)
{
    constexpr int N = Sys::N;
    mcplx kb[4 * N];
    mcplx yt[N];
#pragma unroll 1
    for (int s = 0; s < 6; s++) {
#pragma unroll
        for (int i = 0; i < N; i++) yt[i] = y[i];
#pragma unroll 1
        for (int t = 0; t < 4; t++) {
            const double wt = ck_in[s][t];
            if (wt == 0.0) continue;
            const double hb = h * wt;
            const mcplx* kt = kb + t * N;
#pragma unroll
            for (int i = 0; i < N; i++) yt[i] += hb * kt[i];
        }
        if (s >= 4) {
            const double f0 = ck_fold[s][0], f1 = ck_fold[s][1], f2 = ck_fold[s][2],
                         f3 = ck_fold[s][3];
            mcplx* const a1 = kb + N;
#pragma unroll 1
            for (int i = 0; i < N; i++)
                a1[i] = f0 * kb[i] + f1 * a1[i] + f2 * kb[2 * N + i] + f3 * kb[3 * N + i];
        }
        Sys::f(c, x + ck_a[s] * h, yt, LocalOut<mcplx>{kb + ck_slot[s] * N, ck_w[s], s >= 4});
    }
    const mcplx* a1 = kb + N;
#pragma unroll
    for (int i = 0; i < N; i++) y[i] = y[i] + h * a1[i];
}

// yint's rescaling (module_int.f90:1910-1919, 1952-1961).  |y| is compared through
// |y|^2 against the squared bounds (1e-40, 1e40, both normal doubles): the
// decision can differ from the reference only within rounding of a bound,
// where either choice scales y exactly as the scale count records.
template <int N>
__device__ __forceinline__ void rescale(mcplx* y, int* scale)
{
    constexpr double TINY2 = SC_TINY * SC_TINY, HUGE2 = SC_HUGE * SC_HUGE;
    bool all_small = true, any_big = false;
#pragma unroll
    for (int k = 0; k < N; k++) all_small = all_small && (val(norm2(y[k])) < TINY2);
    if (all_small) {
        (*scale)++;
#pragma unroll
        for (int k = 0; k < N; k++) y[k] = y[k] * SC_HUGE;
    }
#pragma unroll
    for (int k = 0; k < N; k++) any_big = any_big || (val(norm2(y[k])) > HUGE2);
    if (any_big) {
        (*scale)--;
#pragma unroll
        for (int k = 0; k < N; k++) y[k] = y[k] * SC_TINY;
    }
}

// One Cash-Karp step of yint in this build form (the reverse sweep replays
// yint's steps through it, so the replayed states are yint's).
template <class Sys>
__device__ __forceinline__ void yint_step(const Ctx& c, mcplx* y, double x, double h)
{
#if YSG_SMEM_STAGES
    rkck_step_loop<Sys>(c, y, x, h);
#elif YSG_TANGENT || YSG_LOOPED_STEP
    rkck_step_loop_local<Sys>(c, y, x, h);
#else
    rkck_step<Sys>(c, y, x, h);
#endif
}

// module_int.f90:1847-1968 yint
#if YSG_SMEM_STAGES || YSG_TANGENT || YSG_LOOPED_STEP
#undef YSG_YINT_ATTR
#define YSG_YINT_ATTR __noinline__
#else
#define YSG_YINT_ATTR
#endif

template <class Sys>
__device__ YSG_YINT_ATTR void yint(Ctx& cio, int i1, int i2, double r1, double r2, mcplx* yio, int* scale)
{
    if (r2 == r1) return;
#if YSG_SMEM_STAGES
    // a private copy of the context: the caller's lives in memory (its
    // address is passed in), the copy's fields can stay in registers
    Ctx c = cio;
    cd y[Sys::N];
#pragma unroll
    for (int k = 0; k < Sys::N; k++) y[k] = yio[k];
#else
    Ctx& c = cio;
    mcplx* y = yio;
#endif
    const bool up = r2 > r1;
    const Knot* kn = c.kn;
    const int di = up ? 1 : -1;
#if YSG_COUNT_ONLY
    if (c.pfx) {
        // the two end intervals as below, the whole ones between them from
        // the per-omega prefix sums of the same counts
        auto part = [&](int i, double a, double b) -> unsigned {
            if (a == b) return 0u;
            const double nf = floor(fabs(b - a) / steps(c, i));
            return (unsigned)(1 + (int)fmin(nf, 4194304.0));
        };
        unsigned cnt = 0u;
        if (i1 == i2) cnt = part(i1, r1, r2);
        else if (up && i1 < i2)
            cnt = part(i1, r1, kn[i1 + 1].r) + (unsigned)(c.pfx[i2] - c.pfx[i1 + 1]) + part(i2, kn[i2].r, r2);
        else if (!up && i1 > i2)
            cnt = part(i1, r1, kn[i1].r) + (unsigned)(c.pfx[i1] - c.pfx[i2 + 1]) + part(i2, kn[i2 + 1].r, r2);
        c.nst[Sys::CLS] += cnt;
        c.il = i2;
        return;
    }
#endif
    for (int i = i1; up ? (i <= i2) : (i >= i2); i += di) {
        double rr1, rr2;
        if (up) {
            rr1 = (i == i1) ? r1 : kn[i].r;
            rr2 = (i == i2) ? r2 : kn[i + 1].r;
        } else {
            rr1 = (i == i1) ? r1 : kn[i + 1].r;
            rr2 = (i == i2) ? r2 : kn[i].r;
        }
        if (rr1 == rr2) continue;
        c.il = i;
        double drr = steps(c, i);
        const double nf = floor(fabs(rr2 - rr1) / drr);
        // nf is finite and small for omega > 0; the cap only bounds the loop
        int n = 2 + (int)fmin(nf, 4194304.0);
        drr = (rr2 - rr1) / (double)(n - 1);
        c.nst[Sys::CLS] += (unsigned)(n - 1);
        if (YSG_COUNT_ONLY) continue;
        for (int j = 1; j <= n - 1; j++) {
            double rr = __dadd_rn(rr1, __dmul_rn((double)(j - 1), drr));
            yint_step<Sys>(c, y, rr, drr);
            if (scale) rescale<Sys::N>(y, scale);
        }
    }
#if YSG_SMEM_STAGES
#pragma unroll
    for (int k = 0; k < Sys::N; k++) yio[k] = y[k];
    cio.il = c.il;
    cio.nst[Sys::CLS] = c.nst[Sys::CLS];
#endif
}

// The transpose of yint for a linear system (Sys the transposed system, e.g.
// BvecSolidGTr): w <- (M_1 ... M_n)^T w for the steps M_j that
// yint(c, i1, i2, r1, r2) takes, visited in reverse order at the same
// (x, h), with yint's 1e+-20 rescaling of w counted in *scale.  The
// count-only build counts the same steps as the forward integration.
template <class Sys>
__device__ YSG_YINT_ATTR void yint_T(Ctx& cio, int i1, int i2, double r1, double r2, mcplx* wio, int* scale)
{
#if YSG_COUNT_ONLY
    yint<Sys>(cio, i1, i2, r1, r2, wio, scale);     // the same steps, counted
#elif !YSG_SMEM_STAGES
    static_assert(sizeof(Sys) == 0, "yint_T is built in the shared-memory and count-only forms only");
#else
    if (r2 == r1) return;
    Ctx c = cio;
    cd w[Sys::N];
#pragma unroll
    for (int k = 0; k < Sys::N; k++) w[k] = wio[k];
    const bool up = r2 > r1;
    const Knot* kn = c.kn;
    const int di = up ? 1 : -1;
    for (int i = i2; up ? (i >= i1) : (i <= i1); i -= di) {
        double rr1, rr2;
        if (up) {
            rr1 = (i == i1) ? r1 : kn[i].r;
            rr2 = (i == i2) ? r2 : kn[i + 1].r;
        } else {
            rr1 = (i == i1) ? r1 : kn[i + 1].r;
            rr2 = (i == i2) ? r2 : kn[i].r;
        }
        if (rr1 == rr2) continue;
        c.il = i;
        double drr = steps(c, i);
        const double nf = floor(fabs(rr2 - rr1) / drr);
        int n = 2 + (int)fmin(nf, 4194304.0);
        drr = (rr2 - rr1) / (double)(n - 1);
        c.nst[Sys::CLS] += (unsigned)(n - 1);
        for (int j = n - 1; j >= 1; j--) {
            double rr = __dadd_rn(rr1, __dmul_rn((double)(j - 1), drr));
            rkck_step_loop_T<Sys>(c, w, rr, drr);
            if (scale) rescale<Sys::N>(w, scale);
        }
    }
#pragma unroll
    for (int k = 0; k < Sys::N; k++) wio[k] = w[k];
    cio.il = c.il;
    cio.nst[Sys::CLS] = c.nst[Sys::CLS];
#endif
}

// ---------------------------------------------------------------------------
// Start levels, module_start.f90:14-178
// ---------------------------------------------------------------------------
__device__ inline int start_level(const Ctx& c, int l, double w, int i1, int i2, int wt)
{
    const Knot* kn = c.kn;
    int isign = (i2 >= i1) ? 1 : -1;
    double pp = (double)(float)(l * (l + 1)) / __dmul_rn(w, w);
    // q(i) = 1 / v_i^2 - pp / r_i^2, with 1 / v^2 and r^2 formed once per
    // model (knot_derive) by the same rounded operations
    auto q = [&](int i) { return (wt == 1 ? kn[i].inv_b2 : kn[i].inv_a2) - pp / kn[i].r2; };
    int j = i2;
    for (int i = i1; isign == 1 ? i <= i2 : i >= i2; i += isign) {
        double q1 = q(i);
        if (isign == 1) {
            if (q1 > 0.0) { j = max(i1, i - 1); break; }
        } else {
            if (q1 < 0.0) { j = i; break; }
        }
    }
    int is = j;
    int lo = min(i1, i2);
    if (is == lo) return is;
    int j1 = is;
    is = lo;
    double sum = 0.0;
    // each knot's q enters two consecutive intervals: carried from one to the next
    double q1 = q(j1);
    for (int i = j1; i >= lo + 1; i--) {
        const double q2 = q(i - 1);
        if (q1 > 0.0 || q2 > 0.0) {
            sum = 0.0;
        } else {
            const double s1 = sqrt(-q1), s2 = sqrt(-q2);
            double t = __dmul_rn(__dmul_rn(__dmul_rn(0.5, w), __dadd_rn(s1, s2)),
                                 __dsub_rn(kn[i].r, kn[i - 1].r));
            sum = __dadd_rn(sum, t);
        }
        if (sum > TOL_START) { is = i - 1; break; }
        q1 = q2;
    }
    return is;
}

__device__ __forceinline__ int tor_start_level(const Ctx& c, int l, double w, int it)
{
    return start_level(c, l, w, c.mh->noc + 1, it, 1);
}

__device__ inline int sph_start_level(const Ctx& c, int l, double w, int it)
{
    const ModelHdr* mh = c.mh;
    const double aw = -2.00e-3, bw = 2.25e-3, dw = 1.28e-3;
    double wdim = __dmul_rn(w, mh->fre_norm);
    double wsoc = __dadd_rn(aw, __dmul_rn(dw, (double)l));
    int is;
    if (wdim <= wsoc) {
        is = start_level(c, l, w, mh->noc + 1, it, 1);
        if (is == mh->nsl) is = is - 1;
        if (is > mh->noc + 1) return is;
    }
    double wsic = __dadd_rn(aw, __dmul_rn(bw, (double)l));
    if (wdim <= wsic) {
        is = start_level(c, l, w, mh->nic + 1, mh->noc, 2);
        if (is == mh->noc) is = is - 1;
        if (is > mh->nic + 1) return is;
    }
    is = start_level(c, l, w, 2, mh->nic, mh->fic ? 2 : 1);
    if (is == mh->nic) is = is - 1;
    return is;
}

// ---------------------------------------------------------------------------
// Start values
// ---------------------------------------------------------------------------
// module_function.f90:447-490: the ratio j_{l+1}/j_l is the stub x/(2l+3).
__device__ __forceinline__ mcplx sbessj2(int l, mcplx x) { return x / (double)(float)(2 * l + 3); }

// module_function.f90:520-581 bfs: Lentz continued fraction for
// (r dj/dr)/j, or its power series when Re(x^2) <= 0.
__device__ inline mcplx bfs(int l, mcplx xsq, double eps)
{
    if (YSG_COUNT_ONLY) return mk(1.0);     // start values steer no integer decision
    if (val(xsq).x > 0.0) {
        mcplx x = csqrt(xsq);
        int lp1 = l + 1;
        mcplx rx = 2.0 / x;
        double nu = (double)lp1 - 0.5;
        mcplx rj = nu * rx;
        rx = -rx;
        mcplx denom = (nu + 1.0) * rx;
        mcplx numer = denom + 1.0 / rj;
        rj = (rj * numer) / denom;
        int nm1 = 1;
        for (int it = 0; it < 100000; it++) {
            nm1 = nm1 + 1;
            rx = -rx;
            mcplx a3 = (nu + (double)nm1) * rx;
            denom = a3 + 1.0 / denom;
            numer = a3 + 1.0 / numer;
            mcplx ratio = numer / denom;
            rj = rj * ratio;
            if (fabs(val(cabs(ratio)) - 1.0) <= eps) break;
        }
        return rj * x - (double)lp1;
    }
    mcplx f = mk(1.0), fp = mk((double)(float)l), a = mk(1.0);
    double b = (double)(float)(l + l) + 1.0, cc = 2.0, d = (double)(float)l + 2.0;
    for (int it = 0; it < 100000; it++) {
        a = -(a * xsq) / (cc * (b + cc));
        f = f + a;
        fp = fp + a * d;
        if (val(cabs(a * d)) < eps) break;
        cc = cc + 2.0;
        d = d + 2.0;
    }
    return fp / f;
}

// module_function.f90:497-516 bfs_dum: the argument is sqrt(|x^2|).
__device__ __forceinline__ mcplx bfs_dum(int l, mcplx xsq)
{
    mcplx fp = bfs(l, xsq, 1.e-9);
    mreal x = sqrt(cabs(xsq));
    return ((double)l - fp) / x;
}

// module_int.f90:213-250 tor_ystart
__device__ inline void tor_ystart(const Ctx& c, int is, double rr, mcplx* y)
{
    SplPt s = spl_at(c.kn, is, rr);
    mreal rrho = splr(c, s, P_RHO), rmu = splr(c, s, P_MU), rqmu = splr(c, s, P_QMU);
    mcplx cmu = rmu * (1.0 + rqmu * c.lno);
    mcplx cbeta = csqrt(cmu / rrho);
    mcplx arg = (c.omega / cbeta) * rr;
    mcplx ratio = sbessj2(c.llp1, arg);
    y[0] = mk(c.zeta * rr);
    y[1] = c.zeta * (cmu * ((double)(c.ll - 1) - arg * ratio));
}

// module_int.f90:417-489 rad_ystart (GRAV) / rad_ystart_ng
template <bool GRAV>
__device__ inline void rad_ystart(const Ctx& c, int is, double rr, mcplx* y)
{
    SplPt s = spl_at(c.kn, is, rr);
    const Knot* kn = c.kn;
    mreal rrho = splr(c, s, P_RHO), rmu = splr(c, s, P_MU), rqmu = splr(c, s, P_QMU);
    mreal rkappa = splr(c, s, P_KAPPA), rqkappa = splr(c, s, P_QKAPPA);
    mcplx cmu = rmu * (1.0 + rqmu * c.lno);
    mcplx ckappa = rkappa * (1.0 + rqkappa * c.lno);
    mcplx calpha = ckappa + (4.0 * cmu) / 3.0;
    mcplx gamma = GRAV ? c.omega2 + (16.0 * c.mh->pibigg * rrho) / 3.0 : c.omega2;
    gamma = (rrho * gamma) / calpha;
    mcplx arg = gamma * rr;
    mcplx ratio = sbessj2(1, arg);
    y[0] = rr * ratio;
    y[1] = (rr * calpha) * gamma - (4.0 * cmu) * ratio;
}

__device__ __forceinline__ mcplx det2(mcplx a1, mcplx a2, mcplx b1, mcplx b2) { return a1 * b2 - a2 * b1; }

// module_int.f90:1192-1270 sph_solid_start followed by the 14 minors of
// module_int.f90:1451-1485 (sph_minor_solid_start).
__device__ inline void sph_minor_solid_start(const Ctx& c, int is, double rr, mcplx* m)
{
    SplPt s = spl_at(c.kn, is, rr);
    const Knot* kn = c.kn;
    double pib = c.mh->pibigg;
    mreal rrho = splr(c, s, P_RHO), rmu = splr(c, s, P_MU), rqmu = splr(c, s, P_QMU);
    mreal rkappa = splr(c, s, P_KAPPA), rqkappa = splr(c, s, P_QKAPPA);
    mcplx cmu = rmu * (1.0 + rqmu * c.lno);
    mcplx ckappa = rkappa * (1.0 + rqkappa * c.lno);
    mcplx calpha = (ckappa + 1.3333333333 * cmu) / rrho;
    mcplx cbeta = cmu / rrho;
    mcplx tmp1 = c.omega2 / cbeta;
    mcplx tmp2 = (c.omega2 + (5.3333333 * pib) * rrho) / calpha;
    mreal t3 = 2.666666666 * pib * c.zeta * rrho;
    mcplx tmp3 = (t3 * t3) / (calpha * cbeta);
    double ll = (double)c.ll, llp1 = (double)c.llp1;
    mcplx y[6][3];
    double sign = 1.0;
    for (int i = 0; i < 2; i++) {
        mcplx dd = tmp1 - tmp2;
        mcplx gamma = dd * dd + tmp3;
        gamma = 0.5 * (tmp1 + tmp2) + (0.5 * sign) * csqrt(gamma);
        mcplx gamma2 = gamma;
        gamma = csqrt(gamma);
        mcplx zt = ((0.75 * cbeta) * (gamma2 - tmp1)) / (pib * rrho);
        mcplx xi = zt - llp1;
        mcplx args = (gamma2 * rr) * rr;
        mcplx ratio = bfs_dum(c.ll, args);
        mcplx grr = (gamma * rr) * ratio;
        y[0][i] = ll * xi - zt * grr;
        y[1][i] = c.zeta * (xi + grr);
        y[2][i] = -(((4.0 * pib * rrho) * rr) * zt);
        y[3][i] = -((((rrho * calpha) * zt) * rr) * gamma2) +
                  (((2.0 * cmu) * ll) * (ll - 1.0)) * xi / rr +
                  ((2.0 * cmu) * (2.0 * zt + c.zeta2)) * gamma * ratio;
        mcplx y5 = rr * gamma2 + ((2.0 * (ll - 1.0)) * xi) / rr - ((2.0 * (zt + 1.0)) * gamma) * ratio;
        y[4][i] = (cmu * c.zeta) * y5;
        y[5][i] = -(rrho * (c.zeta2 + llp1 * zt));
        sign = -sign;
    }
    y[0][2] = mk(ll);
    y[1][2] = mk(c.zeta);
    y[2][2] = (c.omega2 - (4.0 * pib * rrho * ll) / 3.0) * rr;
    y[3][2] = ((2.0 * ll * (ll - 1.0)) * cmu) / rr;
    y[4][2] = ((2.0 * c.zeta * (ll - 1.0)) * cmu) / rr;
    y[5][2] = ((double)(2 * c.ll + 1) * c.omega2 - (8.0 * pib * ll * (ll - 1.0) * rrho) / 3.0);
    y[5][2] = (0.25 * y[5][2]) / pib;
    // index triples of module_int.f90:1468-1481 (1-based rows)
    const unsigned char idx[14][3] = {{1, 2, 3}, {1, 2, 4}, {1, 2, 5}, {1, 2, 6}, {1, 3, 4},
                                      {1, 3, 5}, {1, 4, 5}, {1, 4, 6}, {1, 5, 6}, {2, 3, 4},
                                      {2, 4, 5}, {2, 4, 6}, {3, 4, 5}, {4, 5, 6}};
#pragma unroll
    for (int q = 0; q < 14; q++) {
        int a = idx[q][0] - 1, b = idx[q][1] - 1, e = idx[q][2] - 1;
        m[q] = y[a][0] * det2(y[b][1], y[e][1], y[b][2], y[e][2]) -
               y[a][1] * det2(y[b][0], y[e][0], y[b][2], y[e][2]) +
               y[a][2] * det2(y[b][0], y[e][0], y[b][1], y[e][1]);
    }
}

__device__ __forceinline__ void minors_of_2col(const mcplx y[4][2], mcplx* m)
{
    m[0] = det2(y[0][0], y[1][0], y[0][1], y[1][1]);
    m[1] = det2(y[0][0], y[2][0], y[0][1], y[2][1]);
    m[2] = det2(y[0][0], y[3][0], y[0][1], y[3][1]);
    m[3] = det2(y[1][0], y[2][0], y[1][1], y[2][1]);
    m[4] = det2(y[2][0], y[3][0], y[2][1], y[3][1]);
}

// 32-bit wrap of the reference's default-integer products
__device__ __forceinline__ int imul32(int a, int b) { return (int)((unsigned)a * (unsigned)b); }

// module_int.f90:1275-1341 sph_solid_start_ng + :1489-1506 minors
__device__ inline void sph_minor_solid_start_ng(const Ctx& c, int is, double rr, mcplx* m)
{
    SplPt s = spl_at(c.kn, is, rr);
    const Knot* kn = c.kn;
    mreal rrho = splr(c, s, P_RHO), rmu = splr(c, s, P_MU), rqmu = splr(c, s, P_QMU);
    mreal rkappa = splr(c, s, P_KAPPA), rqkappa = splr(c, s, P_QKAPPA);
    mcplx cmu = rmu * (1.0 + rqmu * c.lno);
    mcplx ckappa = rkappa * (1.0 + rqkappa * c.lno);
    mcplx calpha = (ckappa + 1.3333333333 * cmu) / rrho;
    mcplx cbeta = cmu / rrho;
    int l = c.ll, lp1 = c.llp1;
    double ll = (double)l;
    mcplx y[4][2];
    mcplx arg = (c.omega * rr) / csqrt(calpha);
    mcplx jl2 = sbessj2(lp1, arg);
    y[0][0] = ll - arg * jl2;
    y[1][0] = mk(c.zeta);
    y[2][0] = (-((((rrho * calpha) * arg) * arg)) +
               (2.0 * cmu) * ((double)imul32(l, l - 1) + (2.0 * arg) * jl2)) / rr;
    y[3][0] = (((2.0 * c.zeta) * cmu) * ((double)(l - 1) - arg * jl2)) / rr;
    arg = (c.omega * rr) / csqrt(cbeta);
    jl2 = sbessj2(lp1, arg);
    y[0][1] = mk(-(double)imul32(l, lp1));
    y[1][1] = -(c.zeta * (double)lp1) + arg * jl2;
    y[2][1] = ((-2.0 * cmu) * ((double)imul32(l, imul32(l, l) - 1) -
                               ((double)imul32(l, lp1) * arg) * jl2)) / rr;
    y[3][1] = ((c.zeta * cmu) * (arg * arg - 2.0 * (double)(imul32(l, l) - 1) - (2.0 * arg) * jl2)) / rr;
    minors_of_2col(y, m);
}

// module_int.f90:1346-1405 sph_fluid_start + :1509-1534 minors
__device__ inline void sph_minor_fluid_start(const Ctx& c, int is, double rr, mcplx* m)
{
    SplPt s = spl_at(c.kn, is, rr);
    const Knot* kn = c.kn;
    double pib = c.mh->pibigg;
    mreal rrho = splr(c, s, P_RHO), rkappa = splr(c, s, P_KAPPA), rqkappa = splr(c, s, P_QKAPPA);
    mcplx ckappa = rkappa * (1.0 + rqkappa * c.lno);
    mcplx calpha = ckappa / rrho;
    mreal gamg = (4.0 * pib * rrho) / 3.0;
    mcplx gamma = ((c.omega2 + 4.0 * gamg) - ((c.zeta2 * gamg) * gamg) * c.omegai2) / calpha;
    mcplx gamma2 = gamma;
    gamma = csqrt(gamma);
    mcplx zt = -c.omega2 / gamg;
    mcplx xi = zt - (double)c.llp1;
    mcplx args = (gamma2 * rr) * rr;
    mcplx ratio = bfs_dum(c.ll, args);
    double ll = (double)c.ll;
    mcplx y[4][2];
    y[0][0] = ll * xi - ((zt * gamma) * rr) * ratio;
    y[1][0] = -(((4.0 * pib * rrho) * rr) * zt);
    y[2][0] = -((((rrho * calpha) * zt) * rr) * gamma2);
    y[3][0] = -(rrho * (c.zeta2 + (double)c.llp1 * zt));
    y[0][1] = mk(ll);
    y[1][1] = (c.omega2 - (4.0 * pib * rrho * ll) / 3.0) * rr;
    y[2][1] = mk(0.0);
    y[3][1] = ((double)(2 * c.ll + 1) * c.omega2 - (8.0 * pib * ll * (ll - 1.0) * rrho) / 3.0);
    y[3][1] = (0.25 * y[3][1]) / pib;
    minors_of_2col(y, m);
}

// module_int.f90:1407-1447 sph_fluid_start_ng (2 components)
__device__ inline void sph_fluid_start_ng(const Ctx& c, int is, double rr, mcplx* y)
{
    SplPt s = spl_at(c.kn, is, rr);
    const Knot* kn = c.kn;
    mreal rrho = splr(c, s, P_RHO), rkappa = splr(c, s, P_KAPPA), rqkappa = splr(c, s, P_QKAPPA);
    mcplx ckappa = rkappa * (1.0 + rqkappa * c.lno);
    mcplx calpha = ckappa / rrho;
    mcplx arg = (c.omega * rr) / csqrt(calpha);
    mcplx ratio = sbessj2(c.llp1, arg);
    y[0] = (double)c.ll - arg * ratio;
    y[1] = (-((rrho * calpha) * arg * arg)) / rr;
}

// ---------------------------------------------------------------------------
// Minor algebra, module_int.f90:1563-1837 (1-based names M(k), S(k), B(k))
// ---------------------------------------------------------------------------
#define YM(k) m[(k) - 1]
#define YS(k) s[(k) - 1]
#define YB(k) b[(k) - 1]

__device__ __forceinline__ void b_solid_start(const mcplx* m, const mcplx* s, mcplx* b)
{
    b[0] = YM(14) * YS(3) - YM(7) * YS(4) - YM(11) * YS(5) - YM(13) * YS(6);
    b[1] = -(YM(14) * YS(2)) - YM(8) * YS(4) - YM(12) * YS(5) + YM(11) * YS(6);
    b[2] = YM(7) * YS(2) + YM(8) * YS(3) + YM(2) * YS(5) + YM(5) * YS(6);
    b[3] = YM(11) * YS(2) + YM(12) * YS(3) - YM(2) * YS(4) + YM(10) * YS(6);
    b[4] = YM(13) * YS(2) - YM(11) * YS(3) - YM(5) * YS(4) - YM(10) * YS(5);
    b[5] = YM(14) * YS(1) - YM(9) * YS(4) + YM(8) * YS(5) - YM(7) * YS(6);
    b[6] = -(YM(7) * YS(1)) + YM(9) * YS(3) + YM(3) * YS(5) + YM(6) * YS(6);
    b[7] = -(YM(11) * YS(1)) - YM(8) * YS(3) - YM(3) * YS(4) - YM(5) * YS(6);
    b[8] = -(YM(13) * YS(1)) + YM(7) * YS(3) - YM(6) * YS(4) + YM(5) * YS(5);
    b[9] = -(YM(8) * YS(1)) - YM(9) * YS(2) + YM(4) * YS(5) - YM(3) * YS(6);
    b[10] = -(YM(12) * YS(1)) + YM(8) * YS(2) - YM(4) * YS(4) + YM(2) * YS(6);
    b[11] = YM(2) * YS(1) + YM(3) * YS(2) + YM(4) * YS(3) - YM(1) * YS(6);
    b[12] = YM(5) * YS(1) + YM(6) * YS(2) - YM(3) * YS(3) + YM(1) * YS(5);
    b[13] = YM(10) * YS(1) - YM(5) * YS(2) + YM(2) * YS(3) - YM(1) * YS(4);
}

__device__ __forceinline__ void b_solid_start_ngcow(const mcplx* m, const mcplx* s, mcplx* b)
{
    b[0] = -(YM(5) * YS(2)) - YM(2) * YS(3) - YM(4) * YS(4);
    b[1] = YM(5) * YS(1) - YM(3) * YS(3) + YM(2) * YS(4);
    b[2] = YM(2) * YS(1) + YM(3) * YS(2) - YM(1) * YS(4);
    b[3] = YM(4) * YS(1) - YM(2) * YS(2) + YM(1) * YS(3);
}

__device__ __forceinline__ void s2f(const mcplx* m1, mcplx* m2)
{
    m2[0] = -m1[5]; m2[1] = -m1[6]; m2[2] = m1[8]; m2[3] = -m1[12]; m2[4] = m1[13];
}
__device__ __forceinline__ void s2f_ngcow(const mcplx* m1, mcplx* m2) { m2[0] = -m1[2]; m2[1] = -m1[4]; }
__device__ __forceinline__ void f2s(const mcplx* m1, mcplx* m2)
{
#pragma unroll
    for (int k = 0; k < 14; k++) m2[k] = mk(0.0);
    m2[0] = m1[0]; m2[1] = m1[1]; m2[3] = m1[2]; m2[9] = -m1[3]; m2[11] = -m1[4];
}
__device__ __forceinline__ void f2s_ngcow(const mcplx* m1, mcplx* m2)
{
#pragma unroll
    for (int k = 0; k < 5; k++) m2[k] = mk(0.0);
    m2[0] = m1[0];
    m2[3] = -m1[1];
}

__device__ __forceinline__ mcplx delta_solid(const mcplx* a, const mcplx* b)
{
#define DA(k) a[(k) - 1]
#define DB(k) b[(k) - 1]
    return -(DA(14) * DB(1)) + 2.0 * (DA(7) * DB(2)) + 2.0 * (DA(11) * DB(3)) + DA(13) * DB(4) +
           2.0 * (DA(8) * DB(5)) + DA(12) * DB(6) - 2.0 * (DA(2) * DB(7)) - 2.0 * (DA(5) * DB(8)) -
           DA(10) * DB(9) + DA(9) * DB(10) - 2.0 * (DA(3) * DB(11)) - DA(6) * DB(12) -
           DA(4) * DB(13) + DA(1) * DB(14);
}
__device__ __forceinline__ mcplx delta_solid_ngcow(const mcplx* a, const mcplx* b)
{
    return DA(5) * DB(1) + 2.0 * (DA(2) * DB(2)) + DA(4) * DB(3) + DA(3) * DB(4) + DA(1) * DB(5);
#undef DA
#undef DB
}

__device__ __forceinline__ void sph_ysol(const mcplx* m, const mcplx* b, mcplx* y)
{
    y[0] = YM(3) * YB(3) + YM(1) * YB(6) + YM(2) * YB(7) + 2.0 * (YM(3) * YB(8)) + YM(4) * YB(9) +
           YM(5) * YB(10) + YM(6) * YB(11) + YM(7) * YB(12) + YM(8) * YB(13) + YM(9) * YB(14);
    y[1] = -(YM(1) * YB(2)) - YM(2) * (2.0 * YB(3) + YB(8)) - YM(3) * YB(4) - YM(4) * YB(5) -
           YM(5) * YB(11) - YM(8) * YB(14) + YM(10) * YB(10) + YM(11) * YB(12) + YM(12) * YB(13);
    y[2] = YM(1) * YB(1) - YM(2) * YB(9) + YM(3) * YB(5) + YM(5) * (YB(8) - YB(3)) -
           YM(6) * YB(4) + YM(7) * YB(14) - YM(10) * YB(7) - YM(11) * YB(13) + YM(13) * YB(12);
    y[3] = YM(2) * YB(1) + YM(5) * YB(2) - YM(7) * YB(4) - YM(8) * YB(5) + YM(10) * YB(6) -
           YM(11) * (YB(3) + 2.0 * YB(8)) - YM(12) * YB(9) - YM(13) * YB(11) + YM(14) * YB(14);
    y[4] = YM(3) * YB(1) - YM(5) * YB(6) + YM(6) * YB(2) + YM(7) * (2.0 * YB(3) + YB(8)) +
           YM(8) * YB(9) - YM(9) * YB(5) + YM(11) * YB(7) + YM(13) * YB(10) - YM(14) * YB(13);
    y[5] = YM(2) * YB(6) - YM(3) * YB(2) + YM(4) * YB(1) + YM(7) * YB(11) +
           YM(8) * (YB(3) - YB(8)) + YM(9) * YB(4) - YM(11) * YB(10) + YM(12) * YB(7) +
           YM(14) * YB(12);
}

// Row k (0, 1 or 2) of sph_ysol as a vector: q . b = sph_ysol(m, b)[k].
__device__ __forceinline__ void sph_ysol_row(const mcplx* m, int k, mcplx* q)
{
#pragma unroll
    for (int j = 0; j < 14; j++) q[j] = mk(0.0);
    if (k == 0) {
        q[2] = YM(3); q[5] = YM(1); q[6] = YM(2); q[7] = 2.0 * YM(3); q[8] = YM(4);
        q[9] = YM(5); q[10] = YM(6); q[11] = YM(7); q[12] = YM(8); q[13] = YM(9);
    } else if (k == 1) {
        q[1] = -YM(1); q[2] = -2.0 * YM(2); q[7] = -YM(2); q[3] = -YM(3); q[4] = -YM(4);
        q[10] = -YM(5); q[13] = -YM(8); q[9] = YM(10); q[11] = YM(11); q[12] = YM(12);
    } else {
        q[0] = YM(1); q[8] = -YM(2); q[4] = YM(3); q[7] = YM(5); q[2] = -YM(5);
        q[3] = -YM(6); q[13] = YM(7); q[6] = -YM(10); q[12] = -YM(11); q[11] = YM(13);
    }
}

// The transpose of b_solid_start in the jump vector: u[s] = w . b(m, e_s),
// so that w . b_solid_start(m, s) = sum_s u[s] s[s].
__device__ __forceinline__ void b_solid_start_T(const mcplx* m, const mcplx* w, mcplx* u)
{
    u[0] = YM(14) * w[5] - YM(7) * w[6] - YM(11) * w[7] - YM(13) * w[8] - YM(8) * w[9] -
           YM(12) * w[10] + YM(2) * w[11] + YM(5) * w[12] + YM(10) * w[13];
    u[1] = -(YM(14) * w[1]) + YM(7) * w[2] + YM(11) * w[3] + YM(13) * w[4] - YM(9) * w[9] +
           YM(8) * w[10] + YM(3) * w[11] + YM(6) * w[12] - YM(5) * w[13];
    u[2] = YM(14) * w[0] + YM(8) * w[2] + YM(12) * w[3] - YM(11) * w[4] + YM(9) * w[6] -
           YM(8) * w[7] + YM(7) * w[8] + YM(4) * w[11] - YM(3) * w[12] + YM(2) * w[13];
    u[3] = -(YM(7) * w[0]) - YM(8) * w[1] - YM(2) * w[3] - YM(5) * w[4] - YM(9) * w[5] -
           YM(3) * w[7] - YM(6) * w[8] - YM(4) * w[10] - YM(1) * w[13];
    u[4] = -(YM(11) * w[0]) - YM(12) * w[1] + YM(2) * w[2] - YM(10) * w[4] + YM(8) * w[5] +
           YM(3) * w[6] + YM(5) * w[8] + YM(4) * w[9] + YM(1) * w[12];
    u[5] = -(YM(13) * w[0]) + YM(11) * w[1] + YM(5) * w[2] + YM(10) * w[3] - YM(7) * w[5] +
           YM(6) * w[6] - YM(5) * w[7] - YM(3) * w[9] + YM(2) * w[10] - YM(1) * w[11];
}

// Row k (0 or 1) of sph_ysol_ngcow as a vector, and the transpose of
// b_solid_start_ngcow in the jump vector (as sph_ysol_row, b_solid_start_T).
__device__ __forceinline__ void sph_ysol_row_ngcow(const mcplx* m, int k, mcplx* q)
{
    if (k == 0) {
        q[0] = mk(0.0); q[1] = YM(1); q[2] = YM(2); q[3] = YM(3);
    } else {
        q[0] = -YM(1); q[1] = mk(0.0); q[2] = YM(4); q[3] = -YM(2);
    }
}

__device__ __forceinline__ void b_solid_start_T_ngcow(const mcplx* m, const mcplx* w, mcplx* u)
{
    u[0] = YM(5) * w[1] + YM(2) * w[2] + YM(4) * w[3];
    u[1] = -(YM(5) * w[0]) + YM(3) * w[2] - YM(2) * w[3];
    u[2] = -(YM(2) * w[0]) - YM(3) * w[1] + YM(1) * w[3];
    u[3] = -(YM(4) * w[0]) + YM(2) * w[1] - YM(1) * w[2];
}

__device__ __forceinline__ void sph_ysol_ngcow(const mcplx* m, const mcplx* b, mcplx* y)
{
    y[0] = YM(1) * YB(2) + YM(2) * YB(3) + YM(3) * YB(4);
    y[1] = -(YM(1) * YB(1)) + YM(4) * YB(3) - YM(2) * YB(4);
    y[2] = -(YM(2) * YB(1)) - YM(4) * YB(2) + YM(5) * YB(4);
    y[3] = -(YM(3) * YB(1)) + YM(2) * YB(2) - YM(5) * YB(3);
}
#undef YM
#undef YS
#undef YB

}  // inline namespace
}  // namespace ysg
#endif  // YSG_ODE_BODY
