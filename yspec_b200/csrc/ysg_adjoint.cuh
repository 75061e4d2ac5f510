// ysg_adjoint.cuh -- reverse-mode (adjoint) sweep of the radial integration.
//
// The gradient of a real loss L with respect to the earth model, for the
// forward solve of ysg_ode.cuh / ysg_solvers.cuh, by the discrete adjoint of
// every operation of a solve: no reference counterpart (the reference has
// no derivatives).  Conventions:
//   - for a complex intermediate z, its adjoint zb satisfies
//     dL = Re(sum zb dz); a linear map w = M z gives zb = M^T wb (plain
//     transpose), a product w = x y gives xb += wb y, yb += wb x;
//   - real model quantities v get real adjoints vb = Re(sum zb dz/dv);
//   - the model enters only through the power-form spline segments
//     c[p][k] of each knot interval (value = c0 + u (c1 + u (c2 + u c3)),
//     u = r - r_i), so the sweep returns dL/dc[i][p][k]: the moments
//     vb_p(r) u^k summed over every point r at which interval i was
//     evaluated.
//
// A Cash-Karp step y1 = y0 + h sum_s c_s k_s, k_s = A(r_s) Y_s is linear in
// y0.  Its adjoint recomputes the stage inputs Y_s from the stored y0, then
// runs the stages backward: Yb_s = A_s^T kb_s (ysg_rhs_adjoint.cuh, tr),
// the coefficient gradients kb_s . (dA/da_e) Y_s (cgrad), the adjoint of the
// coefficient matrix down to the spline values (below), and the stage
// weights kb_t += h b_st Yb_s.  yint's rescaling multiplies the step by
// 1e+-20; the adjoint multiplies by the same factor.
#pragma once
#include "ysg_rhs_adjoint.cuh"

namespace ysg {
inline namespace YSG_VARIANT {

#ifdef __CUDA_ARCH__
__device__ __forceinline__ void grad_add(double* p, double v) { atomicAdd(p, v); }
#else
inline void grad_add(double* p, double v) { *p += v; }
#endif

// dL/dc[i][p][k] for the interval being swept, flushed to the global array
// g ((nknot + 1) x NPARAM x 4 doubles) when the sweep leaves the interval.
struct SegGrad {
    double* g;
    int il;
    double acc[NPARAM][4];
    __device__ void init(double* out)
    {
        g = out;
        il = -1;
        for (int p = 0; p < NPARAM; p++)
            for (int k = 0; k < 4; k++) acc[p][k] = 0.0;
    }
    __device__ void flush()
    {
        if (il < 0) return;
        for (int p = 0; p < NPARAM; p++)
            for (int k = 0; k < 4; k++)
                if (acc[p][k] != 0.0) {
                    grad_add(&g[((size_t)il * NPARAM + p) * 4 + k], acc[p][k]);
                    acc[p][k] = 0.0;
                }
    }
    // vb: dL/dv_p at offset u from the base of interval i
    __device__ void add(int i, double u, const double* vb)
    {
        if (i != il) {
            flush();
            il = i;
        }
        const double u2 = u * u, u3 = u2 * u;
        for (int p = 0; p < NPARAM; p++) {
            const double v = vb[p];
            if (v == 0.0) continue;
            acc[p][0] += v;
            acc[p][1] += v * u;
            acc[p][2] += v * u2;
            acc[p][3] += v * u3;
        }
    }
};

__device__ __forceinline__ double re(cd z) { return z.x; }

// ---------------------------------------------------------------------------
// Adjoints of the coefficient matrices (module_int.f90:134-164, 500-560,
// 676-715): from the entry adjoints s to the adjoints vb of the spline values
// at rr (added to vb).  They restate the forward formulas in the plain form
// (1/(C q) and so on); every derivative is of the same function.
// ---------------------------------------------------------------------------
__device__ inline void tor_amat_adj(const Ctx& c, double rr, const TorCoefBar& s, double* vb)
{
    const Seg& g = c.sg[c.il];
    const double u = rr - g.r0;
    const double rlcon = seg(g, u, P_LCON), rncon = seg(g, u, P_NCON), rqmu = seg(g, u, P_QMU);
    const cd qll = 1.0 + rqmu * c.lno;
    const cd k = 1.0 / (rlcon * qll);                 // a.k
    const double ri = 1.0 / rr;
    // a.s = -omega^2 rho + ri^2 (zeta^2 - 2) N qll
    vb[P_RHO] += re(s.s * (-c.omega2));
    const cd cnb = s.s * (ri * ri * c.zeta2m2);       // adjoint of cncon = N qll
    vb[P_NCON] += re(cnb * qll);
    cd qb = cnb * rncon;
    // a.k = 1 / (L qll)
    vb[P_LCON] += re(s.k * (-k / rlcon));
    qb += s.k * (-k / qll);
    vb[P_QMU] += re(qb * c.lno);
}

template <int KIND>
__device__ inline void solid_amat_adj(const Ctx& c, double rr, const SolidCoefBar& s, double* vb)
{
    const Seg& g = c.sg[c.il];
    const double u = rr - g.r0;
    const double rrho = seg(g, u, P_RHO), racon = seg(g, u, P_ACON), rccon = seg(g, u, P_CCON);
    const double rfcon = seg(g, u, P_FCON), rncon = seg(g, u, P_NCON), rlcon = seg(g, u, P_LCON);
    const double rqmu = seg(g, u, P_QMU), rxlam = seg(g, u, P_XLAM), rxa2 = seg(g, u, P_XA2);
    const cd qaa = 1.0 + rxa2 * c.lno, qff = 1.0 + rxlam * c.lno, qll = 1.0 + rqmu * c.lno;
    const cd cfcon = rfcon * qff;
    const cd k11 = 1.0 / (rccon * qaa), k22 = 1.0 / (rlcon * qll);
    const double ri = 1.0 / rr, ri2 = ri * ri;
    const cd mw2 = -c.omega2;
    // s22 = -omega^2 rho + (zeta^2 (gamma + cncon) - 2 cncon) ri^2
    vb[P_RHO] += re(s.s22 * mw2);
    cd gb = s.s22 * (c.zeta2 * ri2);                 // gamma adjoint
    cd cnb = s.s22 * ((c.zeta2 - 2.0) * ri2);        // cncon adjoint
    if (KIND == 0) {
        vb[P_RHO] += re(s.s11 * mw2);
        gb += s.s11 * (4.0 * ri2) + s.s12 * (-2.0 * c.zeta * ri2);
    } else {
        const double gg = seg(g, u, P_GRAV);
        // s11 = -omega^2 rho + 4 (gamma - rho g r) ri^2, s12 = zeta (rho g r - 2 gamma) ri^2
        vb[P_RHO] += re(s.s11 * mw2) + re(s.s11) * (-4.0 * gg * rr * ri2) + re(s.s12) * (c.zeta * gg * rr * ri2);
        vb[P_GRAV] += re(s.s11) * (-4.0 * rrho * rr * ri2) + re(s.s12) * (c.zeta * rrho * rr * ri2);
        gb += s.s11 * (4.0 * ri2) + s.s12 * (-2.0 * c.zeta * ri2);
    }
    if (KIND == 2) {
        const double pib = c.pib;
        // t31 = -4 pib rho, s13 = -rho (l+1) ri, s23 = rho zeta ri (t33, k33 model-free)
        vb[P_RHO] += re(s.t31) * (-4.0 * pib) + re(s.s13) * (-(double)c.llp1 * ri) + re(s.s23) * (c.zeta * ri);
    }
    // gamma = A qaa - N qll - cfcon^2 k11
    cd cab = gb;
    cnb = cnb - gb;
    cd cfb = gb * (-2.0 * (cfcon * k11));
    cd k11b = gb * (-(cfcon * cfcon)) + s.k11;
    // fc = cfcon k11: t11 = (1 - 2 fc) ri, t12 = zeta ri fc
    const cd fcb = s.t11 * (-2.0 * ri) + s.t12 * (c.zeta * ri);
    cfb += fcb * k11;
    k11b += fcb * cfcon;
    // k11 = 1 / (C qaa), k22 = 1 / (L qll)
    vb[P_CCON] += re(k11b * (-k11 / rccon));
    cd qab = k11b * (-k11 / qaa);
    vb[P_LCON] += re(s.k22 * (-k22 / rlcon));
    cd qlb = s.k22 * (-k22 / qll);
    // cacon = A qaa, cfcon = F qff, cncon = N qll
    vb[P_ACON] += re(cab * qaa);
    qab += cab * racon;
    vb[P_FCON] += re(cfb * qff);
    const cd qfb = cfb * rfcon;
    vb[P_NCON] += re(cnb * qll);
    qlb += cnb * rncon;
    vb[P_XA2] += re(qab * c.lno);
    vb[P_XLAM] += re(qfb * c.lno);
    vb[P_QMU] += re(qlb * c.lno);
}

template <int KIND>
__device__ inline void fluid_amat_adj(const Ctx& c, double rr, const FluidCoefBar& s, double* vb)
{
    const Seg& g = c.sg[c.il];
    const double u = rr - g.r0;
    const double rrho = seg(g, u, P_RHO), rccon = seg(g, u, P_CCON), rxa2 = seg(g, u, P_XA2);
    const cd qaa = 1.0 + rxa2 * c.lno;
    const cd k = 1.0 / (rccon * qaa);                 // cccon
    const double ri = 1.0 / rr, ri2 = ri * ri;
    // k11 = cccon - zeta^2 omega^-2 ri^2 / rho
    const cd zw = c.zeta2 * c.omegai2;
    cd kb = s.k11;
    vb[P_RHO] += re(s.k11 * (zw * (ri2 / (rrho * rrho))));
    // s11 = -omega^2 rho (KIND 0), else with the gravity terms
    if (KIND == 0) {
        vb[P_RHO] += re(s.s11 * (-c.omega2));
    } else {
        const double gg = seg(g, u, P_GRAV);
        const cd gzw = gg * zw;
        // t11 = gzw ri^2 - ri;  s11 = -omega^2 rho + rho g (gzw ri^2 - 4 ri)
        cd gzwb = s.t11 * ri2;
        vb[P_RHO] += re(s.s11 * (-c.omega2 + gg * (gzw * ri2 - 4.0 * ri)));
        vb[P_GRAV] += re(s.s11 * (rrho * (gzw * ri2 - 4.0 * ri)));
        gzwb += s.s11 * (rrho * gg * ri2);
        if (KIND == 2) {
            // t21 = -4 pib rho; s12 = rho (gzw ri - (l+1)) ri; s22 = rho zeta^2 ri^2 omega^-2
            vb[P_RHO] += re(s.t21) * (-4.0 * c.pib);
            vb[P_RHO] += re(s.s12 * (gzw * ri2 - (double)c.llp1 * ri));
            gzwb += s.s12 * (rrho * ri2);
            vb[P_RHO] += re(s.s22 * (zw * ri2));
        }
        // gzw = g zeta^2 omega^-2
        vb[P_GRAV] += re(gzwb * zw);
    }
    // cccon = 1 / (C qaa)
    vb[P_CCON] += re(kb * (-k / rccon));
    const cd qab = kb * (-k / qaa);
    vb[P_XA2] += re(qab * c.lno);
}

// module_int.f90:261-304 rad_amat:
//   t = (1 - 2 F' C'^-1) / r, k = C'^-1, s = -omega^2 rho + 4 (gamma - rho g r) / r^2,
//   gamma = A' - N' - F'^2 C'^-1, with X' = X (1 + q_X lno)
__device__ inline void rad_amat_adj(const Ctx& c, double rr, const RadCoefBar& s, double* vb)
{
    const Seg& g = c.sg[c.il];
    const double u = rr - g.r0;
    const double rrho = seg(g, u, P_RHO), racon = seg(g, u, P_ACON), rccon = seg(g, u, P_CCON);
    const double rfcon = seg(g, u, P_FCON), rncon = seg(g, u, P_NCON), gg = seg(g, u, P_GRAV);
    const double rqmu = seg(g, u, P_QMU), rxlam = seg(g, u, P_XLAM), rxa2 = seg(g, u, P_XA2);
    const cd qaa = 1.0 + rxa2 * c.lno, qff = 1.0 + rxlam * c.lno, qll = 1.0 + rqmu * c.lno;
    const cd cfcon = rfcon * qff;
    const cd k = 1.0 / (rccon * qaa);
    const double ri = 1.0 / rr, ri2 = ri * ri;
    vb[P_RHO] += re(s.s * (-c.omega2)) + re(s.s) * (-4.0 * gg * rr * ri2);
    vb[P_GRAV] += re(s.s) * (-4.0 * rrho * rr * ri2);
    const cd gb = s.s * (4.0 * ri2);
    // gamma = cacon - cncon - cfcon^2 k
    const cd cab = gb, cnb = -gb;
    cd cfb = gb * (-2.0 * (cfcon * k));
    cd kb = gb * (-(cfcon * cfcon)) + s.k;
    // t = (1 - 2 cfcon k) ri
    const cd fcb = s.t * (-2.0 * ri);
    cfb += fcb * k;
    kb += fcb * cfcon;
    vb[P_CCON] += re(kb * (-k / rccon));
    cd qab = kb * (-k / qaa);
    vb[P_ACON] += re(cab * qaa);
    qab += cab * racon;
    vb[P_FCON] += re(cfb * qff);
    const cd qfb = cfb * rfcon;
    vb[P_NCON] += re(cnb * qll);
    const cd qlb = cnb * rncon;
    vb[P_XA2] += re(qab * c.lno);
    vb[P_XLAM] += re(qfb * c.lno);
    vb[P_QMU] += re(qlb * c.lno);
}

// The systems the reverse sweep supports, with their coefficient matrices.
struct TorT {
    using Sys = TorSys;
    using A = TorSysAdj;
    __device__ static TorCoef amat(const Ctx& c, double r) { return tor_amat(c, r); }
    __device__ static void amat_adj(const Ctx& c, double r, const TorCoefBar& s, double* vb) { tor_amat_adj(c, r, s, vb); }
};
struct RadT {
    using Sys = RadSys;
    using A = RadSysAdj;
    __device__ static RadCoef amat(const Ctx& c, double r) { return rad_amat(c, r); }
    __device__ static void amat_adj(const Ctx& c, double r, const RadCoefBar& s, double* vb) { rad_amat_adj(c, r, s, vb); }
};
struct MinorSolidGT {
    using Sys = MinorSolidG;
    using A = MinorSolidGAdj;
    __device__ static SolidCoef amat(const Ctx& c, double r) { return solid_amat<2>(c, r); }
    __device__ static void amat_adj(const Ctx& c, double r, const SolidCoefBar& s, double* vb) { solid_amat_adj<2>(c, r, s, vb); }
};
struct MinorFluidGT {
    using Sys = MinorFluidG;
    using A = MinorFluidGAdj;
    __device__ static FluidCoef amat(const Ctx& c, double r) { return fluid_amat<2>(c, r); }
    __device__ static void amat_adj(const Ctx& c, double r, const FluidCoefBar& s, double* vb) { fluid_amat_adj<2>(c, r, s, vb); }
};
struct BvecSolidGT {
    using Sys = BvecSolidG;
    using A = BvecSolidGAdj;
    __device__ static SolidCoef amat(const Ctx& c, double r) { return solid_amat<2>(c, r); }
    __device__ static void amat_adj(const Ctx& c, double r, const SolidCoefBar& s, double* vb) { solid_amat_adj<2>(c, r, s, vb); }
};
// without self-gravitation: KIND 0 no gravity, 1 Cowling (module_int.f90:874-1110)
template <int KIND>
struct MinorSolidNCT {
    using Sys = MinorSolidNC<KIND>;
    using A = MinorSolidNCAdj;
    __device__ static SolidCoef amat(const Ctx& c, double r) { return solid_amat<KIND>(c, r); }
    __device__ static void amat_adj(const Ctx& c, double r, const SolidCoefBar& s, double* vb) { solid_amat_adj<KIND>(c, r, s, vb); }
};
template <int KIND>
struct MinorFluidNCT {
    using Sys = MinorFluidNC<KIND>;
    using A = MinorFluidNCAdj;
    __device__ static FluidCoef amat(const Ctx& c, double r) { return fluid_amat<KIND>(c, r); }
    __device__ static void amat_adj(const Ctx& c, double r, const FluidCoefBar& s, double* vb) { fluid_amat_adj<KIND>(c, r, s, vb); }
};
template <int KIND>
struct BvecSolidNCT {
    using Sys = BvecSolidNC<KIND>;
    using A = BvecSolidNCAdj;
    __device__ static SolidCoef amat(const Ctx& c, double r) { return solid_amat<KIND>(c, r); }
    __device__ static void amat_adj(const Ctx& c, double r, const SolidCoefBar& s, double* vb) { solid_amat_adj<KIND>(c, r, s, vb); }
};

// Cash-Karp tableau (module_int.f90:2039-2049)
__device__ __forceinline__ double ck_b(int s, int t)
{
    const double b[6][5] = {{0, 0, 0, 0, 0},
                            {0.2, 0, 0, 0, 0},
                            {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0},
                            {0.3, -0.9, 1.2, 0, 0},
                            {-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0},
                            {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0}};
    return b[s][t];
}
__device__ __forceinline__ double ck_c(int s)
{
    const double cc[6] = {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0};
    return cc[s];
}
__device__ __forceinline__ double ck_x(int s)
{
    const double a[6] = {0.0, 0.2, 0.3, 0.6, 1.0, 0.875};
    return a[s];
}

// Adjoint of one Cash-Karp step from y (the state before it) at x with
// step h: on entry yb is the adjoint of the step's result, on exit that of
// y; the model gradient of the step goes to G.
template <class T>
__device__ void rk_step_adj(const Ctx& c, const cd* y, double x, double h, cd* yb, SegGrad& G)
{
    constexpr int N = T::A::N;
    // K holds the stage derivatives k_s while the stage inputs Y_s are
    // formed, then their adjoints; the stage loops stay rolled (one copy of
    // each right-hand side and of its transposes in the code)
    cd Y[6][N], K[6][N];
#pragma unroll 1
    for (int s = 0; s < 6; s++) {
        for (int i = 0; i < N; i++) {
            cd v = y[i];
            for (int t = 0; t < s; t++) v = v + (h * ck_b(s, t)) * K[t][i];
            Y[s][i] = v;
        }
        T::Sys::f(c, x + ck_x(s) * h, Y[s], K[s]);
    }
#pragma unroll 1
    for (int s = 0; s < 6; s++)
        for (int i = 0; i < N; i++) K[s][i] = (h * ck_c(s)) * yb[i];
#pragma unroll 1
    for (int s = 5; s >= 0; s--) {
        const double r = x + ck_x(s) * h;
        const auto a = T::amat(c, r);
        cd Yb[N];
        T::A::tr(a, K[s], Yb);
        typename T::A::Bar sb;
        sb.zero();
        T::A::cgrad(K[s], Y[s], sb);
        double vb[NPARAM];
        for (int p = 0; p < NPARAM; p++) vb[p] = 0.0;
        T::amat_adj(c, r, sb, vb);
        G.add(c.il, r - c.sg[c.il].r0, vb);
        for (int i = 0; i < N; i++) yb[i] = yb[i] + Yb[i];
#pragma unroll 1
        for (int t = 0; t < s; t++) {
            const double w = h * ck_b(s, t);
            for (int i = 0; i < N; i++) K[t][i] = K[t][i] + w * Yb[i];
        }
    }
}

// Work space of one yint sweep: the state before every step, the step's
// radius, size, interval and rescaling factor.  Entry e of an array sits at
// e * st, so the logs of the threads of a launch can be interleaved (st =
// the number of logs, each base pointer offset by its thread's index).
struct StepLog {
    cd* y;            // nmax x LOG_N states
    double* x;        // nmax
    double* h;        // nmax
    int* il;          // nmax
    double* f;        // nmax: factor applied after the step (1, 1e20 or 1e-20)
    int nmax;
    int st;
};

// Entry e of a step log holds its state at (e LOG_N + k) st: every system
// takes LOG_N slots, so legs of different systems can share one log.
constexpr int LOG_N = 14;

// The forward yint of ysg_ode.cuh (same intervals, step counts and
// rescaling: scale counts the rescalings when non-null, as in yint) on y in
// place, every step logged from entry `at` of L on; *ns receives the number
// of steps.  Returns false if they exceed the log.
template <class T>
__device__ __noinline__ bool yint_log(Ctx& c, int i1, int i2, double r1, double r2, cd* y, int* scale,
                                      StepLog& L, int at, int* ns)
{
    constexpr int N = T::A::N;
    static_assert(N <= LOG_N, "log slot too small");
    *ns = 0;
    if (r2 == r1) return true;
    const bool up = r2 > r1;
    const Knot* kn = c.kn;
    const int di = up ? 1 : -1;
    int q = at;
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
        int n = 2 + (int)fmin(nf, 4194304.0);
        drr = (rr2 - rr1) / (double)(n - 1);
        for (int j = 1; j <= n - 1; j++) {
            if (q >= L.nmax) return false;
            double rr = __dadd_rn(rr1, __dmul_rn((double)(j - 1), drr));
            const size_t e = (size_t)q * L.st;
            // streaming stores (evict-first): a log outgrows L2 and is read
            // back only by the reverse pass, so it should not push the
            // threads' stack frames out of L2
#ifdef __CUDA_ARCH__
            for (int k = 0; k < N; k++)
                __stcs(reinterpret_cast<double2*>(L.y + ((size_t)q * LOG_N + k) * L.st),
                       make_double2(y[k].x, y[k].y));
#else
            for (int k = 0; k < N; k++) L.y[((size_t)q * LOG_N + k) * L.st] = y[k];
#endif
            L.x[e] = rr;
            L.h[e] = drr;
            L.il[e] = i;
            yint_step<typename T::Sys>(c, y, rr, drr);
            double f = 1.0;
            if (scale) {
                int sc = 0;
                rescale<N>(y, &sc);
                *scale += sc;
                f = sc > 0 ? SC_HUGE : (sc < 0 ? SC_TINY : 1.0);
            }
            L.f[e] = f;
            q++;
        }
    }
    *ns = q - at;
    return true;
}

// The adjoint of the ns steps logged from entry `at` of L on: yb holds the
// adjoint of their result on entry and that of their starting state on exit.
template <class T>
__device__ __noinline__ void yint_rev(Ctx& c, const StepLog& L, int at, int ns, cd* yb, SegGrad& G)
{
    constexpr int N = T::A::N;
    for (int q = at + ns - 1; q >= at; q--) {
        const size_t e = (size_t)q * L.st;
        c.il = L.il[e];
        const double f = L.f[e];
        if (f != 1.0)
            for (int k = 0; k < N; k++) yb[k] = f * yb[k];
        cd ys[N];
        for (int k = 0; k < N; k++) ys[k] = L.y[((size_t)q * LOG_N + k) * L.st];
        rk_step_adj<T>(c, ys, L.x[e], L.h[e], yb, G);
    }
}

// A yint replayed from its starting state y0 into the log, then reversed:
// yb holds the adjoint of the result on entry and that of y0 on exit.
// Returns false if the steps exceed the log.
template <class T>
__device__ __forceinline__ bool yint_adj(Ctx& c, int i1, int i2, double r1, double r2, const cd* y0, cd* yb,
                                         bool scaled, StepLog& L, SegGrad& G)
{
    constexpr int N = T::A::N;
    if (r2 == r1) return true;
    cd y[N];
    for (int k = 0; k < N; k++) y[k] = y0[k];
    int sc = 0, ns = 0;
    if (!yint_log<T>(c, i1, i2, r1, r2, y, scaled ? &sc : nullptr, L, 0, &ns)) return false;
    yint_rev<T>(c, L, 0, ns, yb, G);
    return true;
}

}  // namespace YSG_VARIANT
}  // namespace ysg
