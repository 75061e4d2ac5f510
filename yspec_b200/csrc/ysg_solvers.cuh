// ysg_solvers.cuh -- two-point boundary-value drivers and source vectors.
//
// Device restatement of module_solver.f90: tor_solver (:25-142),
// rad_solver_ng (:335-441), rad_solver_wg (:446-561), the six sph_solver*
// variants (:640-1740) and source_vector_{tor,rad,sph} (:145-215, :566-627,
// :1747-1847), plus the per-(omega,l) epilogue of yspec.f90:263-400 (output
// type scaling, potential/tilt correction, uu/vv/ww coefficients).
#include "ysg_ode.cuh"
// one copy per build form, as ysg_ode.cuh
#undef YSG_SOLVERS_BODY
#if YSG_TANGENT
#ifndef YSG_SOLVERS_DONE_v_tangent
#define YSG_SOLVERS_DONE_v_tangent
#define YSG_SOLVERS_BODY
#endif
#elif YSG_COUNT_ONLY
#ifndef YSG_SOLVERS_DONE_v_count
#define YSG_SOLVERS_DONE_v_count
#define YSG_SOLVERS_BODY
#endif
#elif YSG_SMEM_STAGES
#ifndef YSG_SOLVERS_DONE_v_smem
#define YSG_SOLVERS_DONE_v_smem
#define YSG_SOLVERS_BODY
#endif
#elif YSG_LOOPED_STEP
#ifndef YSG_SOLVERS_DONE_v_loop
#define YSG_SOLVERS_DONE_v_loop
#define YSG_SOLVERS_BODY
#endif
#else
#ifndef YSG_SOLVERS_DONE_v_local
#define YSG_SOLVERS_DONE_v_local
#define YSG_SOLVERS_BODY
#endif
#endif
// Helpers on the event and plain complex values only, the same in every
// form, so they sit outside the per-form namespaces.
#ifndef YSG_SOLVERS_COMMON
#define YSG_SOLVERS_COMMON
namespace ysg {

__device__ __forceinline__ cd omega_of(const EventDev& ev, int j)
{
    // w = wmin + (j-1)*dw - i*ep, formed without contraction (yspec.f90:261)
    const int k = ev.jofs + (j - 1) * ev.jstride;       // index in the full band
    return mk(__dadd_rn(ev.wmin, __dmul_rn((double)k, ev.dw)), -ev.ep);
}

__device__ __forceinline__ cd out_factor(int out, cd w)
{
    // multiply by i*w (velocity) or -w*w (acceleration), yspec.f90:284-288
    return out == 1 ? imul(w) : (out == 2 ? -(w * w) : mk(1.0));
}

}  // namespace ysg
#endif  // YSG_SOLVERS_COMMON

#ifdef YSG_SOLVERS_BODY

namespace ysg {
inline namespace YSG_VARIANT {

// Rows of the spheroidal response matrices a form computes: the
// shared-memory form and its cost model form only the rows a pair uses
// (sph_solver_g: 0-2, sph_solver_nc: 0-1), the other forms all of them.
constexpr int kSphRows = (YSG_SMEM_STAGES || YSG_COUNT_ONLY) ? 3 : 6;
constexpr int kNcRows = (YSG_SMEM_STAGES || YSG_COUNT_ONLY) ? 2 : 4;

__device__ __forceinline__ double huge_pow(int k)
{
    if (YSG_COUNT_ONLY) return 1.0;
    // huge**k for the integer exponents produced by the rescaling counters
    return k == 0 ? 1.0 : pow(SC_HUGE, (double)k);
}

// module_solver.f90:25-142.  Unit source jumps ss = I (yspec.f90:230-232).
__device__ inline void tor_solver(Ctx& c, double rr, double rs, int ir, int is, mcplx yout[2][2])
{
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    int scale1 = 0, scale2 = 0, scale3 = 0;
    mcplx y1[2], y2[2], y3[2];
    const bool up = rr >= rs;
    int it = up ? is : ir;
    int i1 = tor_start_level(c, c.ll, c.omega.x, it);
    if (i1 == it && i1 > mh->noc + 1) i1 = i1 - 1;
    double rt = kn[i1].r;
    if (i1 == mh->noc + 1) { y1[0] = mk(1.0); y1[1] = mk(0.0); }
    else tor_ystart(c, i1, rt, y1);
    mcplx delta;
    if (up) {
        yint<TorSys>(c, i1, is, rt, rs, y1, &scale1);
        y3[0] = y1[0]; y3[1] = y1[1];
        if (rr != rs) yint<TorSys>(c, is, ir, rs, rr, y3, &scale3);
        y2[0] = mk(1.0); y2[1] = mk(0.0);
        if (rr != kn[mh->nsl].r) yint<TorSys>(c, mh->nsl - 1, ir, kn[mh->nsl].r, rr, y2, &scale2);
        delta = 1.0 / (y2[1] * y3[0] - y2[0] * y3[1]);
        // b = y1(2)*ss(1,i) - y1(1)*ss(2,i); yout(:,i) = -delta*y2*b
        mcplx b0 = y1[1], b1 = -y1[0];
        mcplx dy0 = delta * y2[0], dy1 = delta * y2[1];
        yout[0][0] = -(dy0 * b0); yout[1][0] = -(dy1 * b0);
        yout[0][1] = -(dy0 * b1); yout[1][1] = -(dy1 * b1);
    } else {
        yint<TorSys>(c, i1, ir, rt, rr, y1, &scale1);
        y2[0] = mk(1.0); y2[1] = mk(0.0);
        if (rs != kn[mh->nsl].r) yint<TorSys>(c, mh->nsl - 1, is, kn[mh->nsl].r, rs, y2, &scale2);
        y3[0] = y2[0]; y3[1] = y2[1];
        if (rr != rs) yint<TorSys>(c, is, ir, rs, rr, y3, &scale3);
        delta = 1.0 / (y3[1] * y1[0] - y3[0] * y1[1]);
        mcplx b0 = y2[1], b1 = -y2[0];
        mcplx dy0 = delta * y1[0], dy1 = delta * y1[1];
        yout[0][0] = -(dy0 * b0); yout[1][0] = -(dy1 * b0);
        yout[0][1] = -(dy0 * b1); yout[1][1] = -(dy1 * b1);
    }
    if (scale3 != 0) {
        double f = huge_pow(scale3);
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) yout[a][b] = yout[a][b] * f;
    }
}

// module_solver.f90:335-441 rad_solver_ng (rad_derivs_ng == gravity matrix)
__device__ inline void rad_solver_ng(Ctx& c, double rr, double rs, int ir, int is, mcplx yout[2][2])
{
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    int scale1 = 0, scale2 = 0, scale3 = 0;
    mcplx y1[2], y2[2], y3[2], delta;
    double rt = fmin(0.1 * c.dr, 0.1 * kn[2].r);
    rad_ystart<false>(c, 1, rt, y1);
    const bool up = rr >= rs;
    if (up) {
        yint<RadSys>(c, 1, is, rt, rs, y1, &scale1);
        y2[0] = mk(1.0); y2[1] = mk(0.0);
        if (rr != kn[mh->nknot].r) yint<RadSys>(c, mh->nknot - 1, ir, kn[mh->nknot].r, rr, y2, &scale2);
        y3[0] = y2[0]; y3[1] = y2[1];
        if (rs != rr) yint<RadSys>(c, ir, is, rr, rs, y3, &scale3);
    } else {
        yint<RadSys>(c, 1, ir, rt, rr, y1, &scale1);
        y2[0] = mk(1.0); y2[1] = mk(0.0);
        if (rs != kn[mh->nsl].r) yint<RadSys>(c, mh->nsl - 1, is, kn[mh->nsl].r, rs, y2, &scale2);
        y3[0] = y2[0]; y3[1] = y2[1];
        if (rr != rs) yint<RadSys>(c, is, ir, rs, rr, y3, &scale3);
    }
    delta = y3[1] * y1[0] - y3[0] * y1[1];
    delta = val(cabs(delta)) < 1.0e-100 ? mcplx(mk(0.0)) : 1.0 / delta;
    const mcplx* ya = up ? y1 : y2;   // source-side solution forming b
    const mcplx* yb = up ? y2 : y1;   // solution evaluated at the receiver
    mcplx b0 = ya[1], b1 = -ya[0];
    mcplx dy0 = delta * yb[0], dy1 = delta * yb[1];
    yout[0][0] = -(dy0 * b0); yout[1][0] = -(dy1 * b0);
    yout[0][1] = -(dy0 * b1); yout[1][1] = -(dy1 * b1);
    if (up) {
        if (scale3 != 0) {
            double f = huge_pow(scale3);
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) yout[a][b] = yout[a][b] * f;
        }
    } else {
        // module_solver.f90:433-437 only undoes positive scale3
        for (int k = 0; k < scale3; k++)
            for (int a = 0; a < 2; a++)
                for (int b = 0; b < 2; b++) yout[a][b] = yout[a][b] * SC_HUGE;
    }
}

// Grid of module_model.f90:578-787 (grid_count / make_grid), generated on
// the fly.  visit(k, interval, r) sees 1-based grid index k in increasing
// order; the reverse walk sees the same points from the top down.
struct GridSeg { double a, b; int first; };

__device__ __forceinline__ int grid_segs(double r1, double r2, double rs, double rr, GridSeg* sg,
                                         int* src_after, int* rec_after)
{
    // returns number of segments; *_after = segment index after which the
    // source / receiver point is the last point written (-1 if absent)
    bool ls = (rs > r1 && rs <= r2), lr = (rr > r1 && rr <= r2);
    *src_after = -1;
    *rec_after = -1;
    if (ls && lr) {
        if (rs < rr) {
            sg[0] = {r1, rs, 1}; sg[1] = {rs, rr, 2}; sg[2] = {rr, r2, 2};
            *src_after = 0; *rec_after = 1; return 3;
        } else if (rr < rs) {
            sg[0] = {r1, rr, 1}; sg[1] = {rr, rs, 2}; sg[2] = {rs, r2, 2};
            *rec_after = 0; *src_after = 1; return 3;
        }
        sg[0] = {r1, rs, 1}; sg[1] = {rs, r2, 2};
        *src_after = 0; *rec_after = 0; return 2;
    } else if (ls) {
        sg[0] = {r1, rs, 1}; sg[1] = {rs, r2, 2};
        *src_after = 0; return 2;
    } else if (lr) {
        sg[0] = {r1, rr, 1}; sg[1] = {rr, r2, 2};
        *rec_after = 0; return 2;
    }
    sg[0] = {r1, r2, 1};
    return 1;
}

__device__ __forceinline__ int seg_npts(const GridSeg& s, double drr)
{
    return (int)floor((s.b - s.a) / drr) + 2;
}

// module_solver.f90:446-561 rad_solver_wg.  The main program does not use
// the potential (yspec.f90:277-281); with pot non-null it is formed as
// there (:534-554, pout(1, i) for the two unit sources i): rr times the
// trapezoid sum over grid points 1 .. irr of -4 pibigg ys(1) / r, the
// value at the first point taken as zero.  ys is -delta y1s b_below at
// points up to the source and -delta y2s b_above beyond it, so the sum is
// collected on the two walks as S1 (over y1s) and S2 (over y2s) and
// combined at the end.
__device__ inline void rad_solver_wg(Ctx& c, double rr, double rs, mcplx yout[2][2], mcplx* pot = nullptr)
{
    if (YSG_COUNT_ONLY) pot = nullptr;              // the cost model counts steps only
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    const double drr = c.dr;
    // pass 1: grid size and source / receiver indices
    int ngrid = 0, iss = 0, irr = 0;
    for (int i = 1; i <= mh->nknot - 1; i++) {
        double r1 = kn[i].r, r2 = kn[i + 1].r;
        if (r1 == r2) continue;
        GridSeg sg[3];
        int sa, ra;
        int ns = grid_segs(r1, r2, rs, rr, sg, &sa, &ra);
        for (int q = 0; q < ns; q++) {
            ngrid += seg_npts(sg[q], drr) - (sg[q].first - 1);
            if (q == sa) iss = ngrid;
            if (q == ra) irr = ngrid;
        }
    }
    // pass 2: upward from rt through grid points 2..iss
    mcplx y1[2], yrec[2] = {mk(0.0), mk(0.0)};
    mcplx s1 = mk(0.0), s2 = mk(0.0), g1_iss = mk(0.0), g2_next = mk(0.0);
    double r_iss = 0.0, r_next = 0.0;
    bool have_rec = false;
    {
        int k = 0, iprev = 0;
        double rprev = 0.0;
        mcplx gprev = mk(0.0);                       // y1s(1) / r at the previous point
        bool started = false;
        for (int i = 1; i <= mh->nknot - 1 && k < iss; i++) {
            double r1 = kn[i].r, r2 = kn[i + 1].r;
            if (r1 == r2) continue;
            GridSeg sg[3];
            int sa, ra;
            int ns = grid_segs(r1, r2, rs, rr, sg, &sa, &ra);
            for (int q = 0; q < ns && k < iss; q++) {
                int np = seg_npts(sg[q], drr);
                double drt = (sg[q].b - sg[q].a) / (double)(np - 1);
                for (int jj = sg[q].first; jj <= np && k < iss; jj++) {
                    k++;
                    double rk = __dadd_rn(sg[q].a, __dmul_rn((double)(jj - 1), drt));
                    if (k == 2) {
                        double rt = fmin(0.1 * drr, 0.1 * rk);
                        rad_ystart<true>(c, 1, rt, y1);
                        yint<RadSys>(c, 1, i, rt, rk, y1, nullptr);
                        started = true;
                    } else if (k > 2) {
                        yint<RadSys>(c, iprev, i, rprev, rk, y1, nullptr);
                    }
                    if (started && k == irr) { yrec[0] = y1[0]; yrec[1] = y1[1]; have_rec = true; }
                    if (pot && k >= 2) {
                        const mcplx g = y1[0] / rk;
                        if (k <= irr) s1 = s1 + (0.5 * (rk - rprev)) * (gprev + g);
                        if (k == iss) { g1_iss = g; r_iss = rk; }
                        gprev = g;
                    }
                    iprev = i;
                    rprev = rk;
                }
            }
        }
    }
    // pass 3: downward from grid point ngrid to iss
    mcplx y2[2] = {mk(1.0), mk(0.0)};
    {
        int k = ngrid + 1, iprev = 0;
        double rprev = 0.0;
        for (int i = mh->nknot - 1; i >= 1 && k > iss; i--) {
            double r1 = kn[i].r, r2 = kn[i + 1].r;
            if (r1 == r2) continue;
            GridSeg sg[3];
            int sa, ra;
            int ns = grid_segs(r1, r2, rs, rr, sg, &sa, &ra);
            for (int q = ns - 1; q >= 0 && k > iss; q--) {
                int np = seg_npts(sg[q], drr);
                double drt = (sg[q].b - sg[q].a) / (double)(np - 1);
                for (int jj = np; jj >= sg[q].first && k > iss; jj--) {
                    k--;
                    double rk = __dadd_rn(sg[q].a, __dmul_rn((double)(jj - 1), drt));
                    if (k < ngrid) yint<RadSys>(c, iprev, i, rprev, rk, y2, nullptr);
                    if (k == irr && irr > iss) { yrec[0] = y2[0]; yrec[1] = y2[1]; have_rec = true; }
                    if (pot && k > iss) {
                        const mcplx g = y2[0] / rk;
                        // segment [k, k + 1] within [1, irr], above the source
                        if (k < ngrid && k + 1 <= irr) s2 = s2 + (0.5 * (rprev - rk)) * (g + g2_next);
                        g2_next = g;
                        r_next = rk;
                    }
                    iprev = i;
                    rprev = rk;
                }
            }
        }
    }
    (void)have_rec;
    mcplx delta = 1.0 / (y2[1] * y1[0] - y2[0] * y1[1]);
    mcplx b0, b1;
    if (irr <= iss) { b0 = y2[1]; b1 = -y2[0]; }
    else { b0 = y1[1]; b1 = -y1[0]; }
    mcplx dy0 = delta * yrec[0], dy1 = delta * yrec[1];
    yout[0][0] = -(dy0 * b0); yout[1][0] = -(dy1 * b0);
    yout[0][1] = -(dy0 * b1); yout[1][1] = -(dy1 * b1);
    if (pot) {
        // the segment across the source, [iss, iss + 1]
        if (iss + 1 <= irr && iss + 1 <= ngrid) {
            s1 = s1 + (0.5 * (r_next - r_iss)) * g1_iss;
            s2 = s2 + (0.5 * (r_next - r_iss)) * g2_next;
        }
        // pout(1, i) = rr (-4 pibigg) (-delta) (b_below_i S1 + b_above_i S2)
        const mcplx f = (rr * (4.0 * c.mh->pibigg)) * delta;
        pot[0] = f * (y2[1] * s1 + y1[1] * s2);
        pot[1] = f * (-(y2[0] * s1) - y1[0] * s2);
    }
}

// Spheroidal solve with self-gravitation: sph_solver (:640-823) and
// sph_solver_fic (:1203-1382).  yout[6][4] holds the responses to unit
// jumps in components 1, 2, 4, 5 (yspec.f90:234-238).  `rows` (bit k for
// yout[k]) names the rows the caller uses; the shared-memory form computes
// only those (rows 0-2) and leaves the others zero, the other forms compute
// all six.
__device__ inline void sph_solver_g(Ctx& c, double rr, double rs, int ir, int is,
                                    mcplx yout[kSphRows][4], int rows = 0x3f)
{
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    const bool fic = mh->fic != 0;
    int scale1 = 0, scale2 = 0, scale3 = 0;
    mcplx ms1[14], ms2[14], ms3[14], mf[5];
    const bool up = rr >= rs;
    const int it = up ? is : ir;
    const double rtop = up ? rs : rr;
    int i1 = sph_start_level(c, c.ll, c.omega.x, it);
    double rt = kn[i1].r;
    if (i1 == 1 && (up || fic)) rt = fmin(0.1 * c.dr, 0.1 * kn[2].r);
    if (i1 >= it) { i1 = it - 1; rt = kn[i1].r; }
    if (i1 <= mh->nic) {
        if (fic) {
            // A fluid inner core starts from the fluid minor on both branches.
            // The reference's receiver-below-source branch of sph_solver_fic
            // (:1323-1332) starts a solid minor there instead; with mu = 0 its
            // shear wavenumber is infinite and bfs's continued fraction never
            // converges, so the reference does not return for these pairs.
            // The receiver-above branch's fluid start (:1252-1256) is taken for both.
            sph_minor_fluid_start(c, i1, rt, mf);
            yint<MinorFluidG>(c, i1, mh->noc, rt, kn[mh->noc].r, mf, &scale1);
        } else {
            sph_minor_solid_start(c, i1, rt, ms1);
            yint<MinorSolidG>(c, i1, mh->nic, rt, kn[mh->nic].r, ms1, &scale1);
            s2f(ms1, mf);
            yint<MinorFluidG>(c, mh->nic + 1, mh->noc, kn[mh->nic].r, kn[mh->noc].r, mf, &scale1);
        }
        f2s(mf, ms1);
        yint<MinorSolidG>(c, mh->noc + 1, it, kn[mh->noc + 1].r, rtop, ms1, &scale1);
    } else if (i1 <= mh->noc) {
        sph_minor_fluid_start(c, i1, rt, mf);
        yint<MinorFluidG>(c, i1, mh->noc, rt, kn[mh->noc].r, mf, &scale1);
        f2s(mf, ms1);
        yint<MinorSolidG>(c, mh->noc + 1, it, kn[mh->noc + 1].r, rtop, ms1, &scale1);
    } else if (i1 <= mh->nsl) {
        sph_minor_solid_start(c, i1, rt, ms1);
        yint<MinorSolidG>(c, i1, it, rt, rtop, ms1, &scale1);
    }
#pragma unroll
    for (int k = 0; k < 14; k++) ms3[k] = ms1[k];
    if (up) { if (rr > rs) yint<MinorSolidG>(c, is, ir, rs, rr, ms3, &scale3); }
    else { if (rs > rr) yint<MinorSolidG>(c, ir, is, rr, rs, ms3, &scale3); }
    const int ibot = up ? ir : is;
    const double rbot = up ? rr : rs;
    if (mh->ocean) {
        mcplx mf2[5] = {mk(1.0), mk(0.0), mk(0.0), mk(0.0), mk(0.0)};
        yint<MinorFluidG>(c, mh->nknot - 1, mh->nsl + 1, kn[mh->nknot].r, kn[mh->nsl + 1].r, mf2, &scale2);
        f2s(mf2, ms2);
        yint<MinorSolidG>(c, mh->nsl, ibot, kn[mh->nsl].r, rbot, ms2, &scale2);
    } else {
#pragma unroll
        for (int k = 0; k < 14; k++) ms2[k] = mk(0.0);
        ms2[0] = mk(1.0);
        yint<MinorSolidG>(c, up ? mh->nknot - 1 : mh->nknot, ibot, kn[mh->nknot].r, rbot, ms2, &scale2);
    }
    mcplx delta = delta_solid(ms3, ms2);
    const int jump[4] = {0, 1, 3, 4};
#if YSG_SMEM_STAGES || YSG_COUNT_ONLY
    // Row k of the responses to the four jumps is ys_k,i = q_k . Phi b_i:
    // Phi the b-vector propagator from the source to the receiver, b_i the
    // start vector of jump i (b_solid_start of the minor at the source end)
    // and q_k row k of sph_ysol (the minor at the receiver end).  One
    // backward integration of the transposed system per needed row,
    // w_k = Phi^T q_k, gives ys_k,i = w_k . b_i for all four jumps at once,
    // in place of four forward b-vector integrations.  The same quantity
    // as the loop below, different only in rounding.
    {
        const mcplx* mq = up ? ms2 : ms1;
        const mcplx* mb = up ? ms1 : ms2;
        unsigned nrow = 0;
        for (int k = 0; k < kSphRows; k++) {
            if (!((rows >> k) & 1)) {
                for (int i = 0; i < 4; i++) yout[k][i] = mk(0.0);
                continue;
            }
            nrow++;
#if YSG_COUNT_ONLY
            // the rows integrate the same span: one pass counts for each
            if (nrow == 1) yint_T<BvecSolidGTr>(c, is, ir, rs, rr, nullptr, nullptr);
            continue;
#endif
            mcplx w[14], u[6];
            sph_ysol_row(mq, k, w);
            int sw = 0;
            yint_T<BvecSolidGTr>(c, is, ir, rs, rr, w, &sw);
            b_solid_start_T(mb, w, u);
            const double f = huge_pow(scale3 - sw);
            for (int i = 0; i < 4; i++) yout[k][i] = ((-u[jump[i]]) / delta) * f;
        }
        if (YSG_COUNT_ONLY) c.nst[BvecSolidGTr::CLS] *= nrow;
    }
#else
    (void)rows;
    for (int i = 0; i < 4; i++) {
        mcplx s[6] = {mk(0.0), mk(0.0), mk(0.0), mk(0.0), mk(0.0), mk(0.0)};
        s[jump[i]] = mk(1.0);
        int scale4 = 0;
        mcplx b[14], ys[6];
        if (up) {
            b_solid_start(ms1, s, b);
            yint<BvecSolidG>(c, is, ir, rs, rr, b, &scale4);
            sph_ysol(ms2, b, ys);
            for (int k = 0; k < 6; k++) ys[k] = (-ys[k]) / delta;
        } else {
            b_solid_start(ms2, s, b);
            for (int k = 0; k < 14; k++) b[k] = (-b[k]) / delta;
            yint<BvecSolidG>(c, is, ir, rs, rr, b, &scale4);
            sph_ysol(ms1, b, ys);
        }
        double f = huge_pow(scale3 - scale4);
        for (int k = 0; k < 6; k++) yout[k][i] = ys[k] * f;
    }
#endif
}

// No gravity (KIND 0) / Cowling (KIND 1): sph_solver_ng (:827-1010),
// sph_solver_cow (:1014-1195), sph_solver_ng_fic (:1386-1562),
// sph_solver_cow_fic (:1568-1740).  yout[4][4], ss = I (yspec.f90:240-243).
// The shared-memory form computes only rows 0 and 1 (the ones the pair
// uses) and leaves rows 2 and 3 zero.
template <int KIND>
__device__ inline void sph_solver_nc(Ctx& c, double rr, double rs, int ir, int is, mcplx yout[kNcRows][4])
{
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    const bool fic = mh->fic != 0;
    int scale1 = 0, scale2 = 0, scale3 = 0;
    mcplx ms1[5], ms2[5], ms3[5], mf[2];
    const bool up = rr >= rs;
    const int it = up ? is : ir;
    const double rtop = up ? rs : rr;
    int i1 = sph_start_level(c, c.ll, c.omega.x, it);
    double rt = kn[i1].r;
    if (i1 == 1 && (up || fic)) rt = fmin(0.1 * c.dr, 0.1 * kn[2].r);
    if (i1 >= it) { i1 = it - 1; rt = kn[i1].r; }
    if (i1 <= mh->nic) {
        if (fic) {
            sph_fluid_start_ng(c, i1, rt, mf);
            yint<MinorFluidNC<KIND>>(c, i1, mh->noc, rt, kn[mh->noc].r, mf, &scale1);
        } else {
            sph_minor_solid_start_ng(c, i1, rt, ms1);
            yint<MinorSolidNC<KIND>>(c, i1, mh->nic, rt, kn[mh->nic].r, ms1, &scale1);
            s2f_ngcow(ms1, mf);
            yint<MinorFluidNC<KIND>>(c, mh->nic + 1, mh->noc, kn[mh->nic].r, kn[mh->noc].r, mf, &scale1);
        }
        f2s_ngcow(mf, ms1);
        yint<MinorSolidNC<KIND>>(c, mh->noc + 1, it, kn[mh->noc + 1].r, rtop, ms1, &scale1);
    } else if (i1 <= mh->noc) {
        sph_fluid_start_ng(c, i1, rt, mf);
        yint<MinorFluidNC<KIND>>(c, i1, mh->noc, rt, kn[mh->noc].r, mf, &scale1);
        f2s_ngcow(mf, ms1);
        yint<MinorSolidNC<KIND>>(c, mh->noc + 1, it, kn[mh->noc + 1].r, rtop, ms1, &scale1);
    } else if (i1 <= mh->nsl) {
        sph_minor_solid_start_ng(c, i1, rt, ms1);
        yint<MinorSolidNC<KIND>>(c, i1, it, rt, rtop, ms1, &scale1);
    }
#pragma unroll
    for (int k = 0; k < 5; k++) ms3[k] = ms1[k];
    if (up) { if (rr > rs) yint<MinorSolidNC<KIND>>(c, is, ir, rs, rr, ms3, &scale3); }
    else { if (rs > rr) yint<MinorSolidNC<KIND>>(c, ir, is, rr, rs, ms3, &scale3); }
    const int ibot = up ? ir : is;
    const double rbot = up ? rr : rs;
    if (mh->ocean) {
        mcplx mf2[2] = {mk(1.0), mk(0.0)};
        yint<MinorFluidNC<KIND>>(c, mh->nknot - 1, mh->nsl + 1, kn[mh->nknot].r, kn[mh->nsl + 1].r, mf2, &scale2);
        f2s_ngcow(mf2, ms2);
        yint<MinorSolidNC<KIND>>(c, mh->nsl, ibot, kn[mh->nsl].r, rbot, ms2, &scale2);
    } else {
#pragma unroll
        for (int k = 0; k < 5; k++) ms2[k] = mk(0.0);
        ms2[0] = mk(1.0);
        yint<MinorSolidNC<KIND>>(c, mh->nknot, ibot, kn[mh->nknot].r, rbot, ms2, &scale2);
    }
    mcplx delta = delta_solid_ngcow(ms3, ms2);
#if YSG_SMEM_STAGES || YSG_COUNT_ONLY
    // rows 0 and 1 from backward integrations of the transposed system, as
    // in sph_solver_g (the receiver-above branch divides by delta after the
    // integration, the other negates and divides the start vector)
    {
#if YSG_COUNT_ONLY
        yint_T<BvecSolidNCTr<KIND>>(c, is, ir, rs, rr, nullptr, nullptr);
        c.nst[BvecSolidNCTr<KIND>::CLS] *= 2u;
#else
        const mcplx* mq = up ? ms2 : ms1;
        const mcplx* mb = up ? ms1 : ms2;
        const mcplx sg = up ? mk(1.0) : mk(-1.0);
        for (int k = 0; k < 2; k++) {
            mcplx w[4], u[4];
            sph_ysol_row_ngcow(mq, k, w);
            int sw = 0;
            yint_T<BvecSolidNCTr<KIND>>(c, is, ir, rs, rr, w, &sw);
            b_solid_start_T_ngcow(mb, w, u);
            const double f = huge_pow(scale3 - sw);
            for (int i = 0; i < 4; i++) yout[k][i] = ((sg * u[i]) / delta) * f;
        }
#endif
    }
#else
    for (int i = 0; i < 4; i++) {     // see sph_solver_g
        mcplx s[4] = {mk(0.0), mk(0.0), mk(0.0), mk(0.0)};
        s[i] = mk(1.0);
        int scale4 = 0;
        mcplx b[4], ys[4];
        if (up) {
            b_solid_start_ngcow(ms1, s, b);
            yint<BvecSolidNC<KIND>>(c, is, ir, rs, rr, b, &scale4);
            sph_ysol_ngcow(ms2, b, ys);
            for (int k = 0; k < 4; k++) ys[k] = ys[k] / delta;
        } else {
            b_solid_start_ngcow(ms2, s, b);
            for (int k = 0; k < 4; k++) b[k] = (-b[k]) / delta;
            yint<BvecSolidNC<KIND>>(c, is, ir, rs, rr, b, &scale4);
            sph_ysol_ngcow(ms1, b, ys);
        }
        double f = huge_pow(scale3 - scale4);
        for (int k = 0; k < 4; k++) yout[k][i] = ys[k] * f;
    }
#endif
}

// ---------------------------------------------------------------------------
// Source vectors
// ---------------------------------------------------------------------------
// module_solver.f90:145-215 (svt(:,1) and svt(:,2))
__device__ inline void source_vector_tor(const Ctx& c, int is, double rs, const double* mm,
                                         mcplx svt[5][2])
{
    SplPt s = spl_at(c.kn, is, rs);
    mreal rlcon = splr(c, s, P_LCON), rqmu = splr(c, s, P_QMU);
    mcplx clcon = rlcon * (1.0 + rqmu * c.lno);
    for (int i = 0; i < 5; i++) svt[i][0] = svt[i][1] = mk(0.0);
    if (c.ll >= 1) {
        svt[1][0] = ((0.5 * rs) * mk(-mm[2], mm[1])) / clcon;
        svt[3][0] = ((0.5 * rs) * mk(mm[2], mm[1])) / clcon;
    }
    if (c.ll >= 2) {
        svt[0][1] = (0.25 * c.szeta2m2) * mk(2.0 * mm[4], -mm[3] + mm[5]);
        svt[4][1] = (0.25 * c.szeta2m2) * mk(2.0 * mm[4], mm[3] - mm[5]);
    }
    cd den = (imul(c.omega) * rs) * rs;
    for (int i = 0; i < 5; i++) {
        svt[i][0] = (c.nu * svt[i][0]) / den;
        svt[i][1] = (c.nu * svt[i][1]) / den;
    }
}

// module_solver.f90:566-627
__device__ inline void source_vector_rad(const Ctx& c, int is, double rs, const double* mm, mcplx s0[2])
{
    SplPt s = spl_at(c.kn, is, rs);
    mreal rccon = splr(c, s, P_CCON), rfcon = splr(c, s, P_FCON);
    mreal rxa2 = splr(c, s, P_XA2), rxlam = splr(c, s, P_XLAM);
    mcplx cccon = 1.0 / (rccon * (1.0 + rxa2 * c.lno));
    mcplx cfcon = rfcon * (1.0 + rxlam * c.lno);
    s0[0] = (rs * mm[0]) * cccon;
    s0[1] = (-mm[3] - mm[5]) + ((2.0 * mm[0]) * cfcon) * cccon;
    cd den = (imul(c.omega) * rs) * rs;
    s0[0] = (c.nu * s0[0]) / den;
    s0[1] = (c.nu * s0[1]) / den;
}

// module_solver.f90:1747-1847.  qaa, qff and qll are declared real(dp)
// there (:1771-1772), so only Re(1 + q*lno) enters the spheroidal source.
__device__ inline void source_vector_sph(const Ctx& c, int is, double rs, const double* mm,
                                         mcplx svs[5][6])
{
    SplPt s = spl_at(c.kn, is, rs);
    const Knot* kn = c.kn;
    mreal rlcon = splr(c, s, P_LCON), rccon = splr(c, s, P_CCON), rfcon = splr(c, s, P_FCON);
    mreal rqmu = splr(c, s, P_QMU), rxlam = splr(c, s, P_XLAM), rxa2 = splr(c, s, P_XA2);
    mreal qaa = 1.0 + rxa2 * c.lno.x;
    mreal qff = 1.0 + rxlam * c.lno.x;
    mreal qll = 1.0 + rqmu * c.lno.x;
    mreal cccon = 1.0 / (rccon * qaa);
    mreal cfcon = rfcon * qff, clcon = rlcon * qll;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 6; j++) svs[i][j] = mk(0.0);
    double z = c.zeta;
    if (c.ll != 1) svs[0][4] = (0.25 * c.szeta2m2) * mk(-mm[3] + mm[5], -2.0 * mm[4]);
    svs[1][1] = ((0.5 * rs) * mk(mm[1], mm[2])) / clcon;
    svs[2][0] = mk(((rs * mm[0]) * cccon));
    svs[2][3] = mk((-mm[3] - mm[5]) + ((2.0 * mm[0]) * cfcon) * cccon);
    svs[2][4] = mk((0.5 * z) * (mm[3] + mm[5]) - ((z * mm[0]) * cfcon) * cccon);
    svs[3][1] = ((0.5 * rs) * mk(-mm[1], mm[2])) / clcon;
    if (c.ll != 1) svs[4][4] = (0.25 * c.szeta2m2) * mk(-mm[3] + mm[5], 2.0 * mm[4]);
    cd den = (imul(c.omega) * rs) * rs;
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 6; j++) svs[i][j] = (c.nu * svs[i][j]) / den;
}

// ---------------------------------------------------------------------------
// One (omega_j, l) pair: yspec.f90:259-400.  coef = uu(1:5), vv(1:5), ww(1:5).
// ---------------------------------------------------------------------------
// grav(ir), the knot value the potential / tilt correction uses
// (yspec.f90:388-391)
__device__ __forceinline__ mreal grav_at_receiver(const Ctx& c, const EventDev& ev)
{
#if YSG_TANGENT
    return mreal(ev.grav_ir, c.dkn[ev.ir].v[P_GRAV][0]);
#else
    (void)c;
    return ev.grav_ir;
#endif
}

// l == 0: radial mode, yspec.f90:263-293
__device__ inline void pair_radial(Ctx& c, const EventDev& ev, int j, mcplx* coef)
{
    cd w = omega_of(ev, j);
    set_l(c, 0);
    set_omega(c, w);
    mcplx sr0[2], yrad[2][2];
    source_vector_rad(c, ev.is, ev.rs, ev.mm, sr0);
    alpha_steps(c);
    mcplx u3;
    if (ev.pot) {
        // the potential at the receiver (module_solver.f90:534-554); no
        // gravity, no potential
        mcplx ph[2] = {mk(0.0), mk(0.0)};
        if (ev.grav != 0) rad_solver_wg(c, ev.rr, ev.rs, yrad, ph);
        u3 = (sr0[0] * ph[0] + sr0[1] * ph[1]) / ev.rr;
    } else {
        if (ev.grav == 0) rad_solver_ng(c, ev.rr, ev.rs, ev.ir, ev.is, yrad);
        else rad_solver_wg(c, ev.rr, ev.rs, yrad);
        u3 = (sr0[0] * yrad[0][0] + sr0[1] * yrad[0][1]) / ev.rr;
    }
    if (ev.out != 0) u3 = out_factor(ev.out, w) * u3;
    for (int q = 0; q < NCOEF; q++) coef[q] = mk(0.0);
    coef[2] = u3;
}

// l >= 2: toroidal part, yspec.f90:301-316 -> ww(1:5)
__device__ inline void pair_toroidal(Ctx& c, const EventDev& ev, int l, int j, mcplx* ww)
{
    if (ev.pot) {                                     // toroidal motion carries no potential
        for (int q = 0; q < 5; q++) ww[q] = mk(0.0);
        return;
    }
    cd w = omega_of(ev, j);
    set_l(c, l);
    set_omega(c, w);
    mcplx svt[5][2], ytor[2][2];
    source_vector_tor(c, ev.is, ev.rs, ev.mm, svt);
    tor_solver(c, ev.rr, ev.rs, ev.ir, ev.is, ytor);
    if (ev.out != 0) {
        cd f = out_factor(ev.out, w);
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) ytor[a][b] = f * ytor[a][b];
    }
    double zeta = (double)sqrtf((float)(l * (l + 1)));   // yspec.f90:255 (FP32)
    double zr = zeta * ev.rr;
    for (int q = 0; q < 5; q++) ww[q] = (svt[q][0] * ytor[0][0] + svt[q][1] * ytor[0][1]) / zr;
}

// l >= 1: spheroidal part, yspec.f90:344-400 -> uu(1:5), vv(1:5)
__device__ inline void pair_spheroidal(Ctx& c, const EventDev& ev, int l, int j, mcplx* uu, mcplx* vv)
{
    cd w = omega_of(ev, j);
    set_l(c, l);
    set_omega(c, w);
    alpha_steps(c);
    mcplx ysph[kSphRows][4];
    if (ev.grav == 2) {
        // the rows of the responses used below: the potential (row 2) alone,
        // or the two displacement rows, with row 2 for the tilt and
        // potential correction of the acceleration
        const int rows = ev.pot ? 0x4 : ((ev.out == 2 && ev.cor != 0) ? 0x7 : 0x3);
        sph_solver_g(c, ev.rr, ev.rs, ev.ir, ev.is, ysph, rows);
    } else {
        mcplx yng[kNcRows][4];
        if (ev.grav == 1) sph_solver_nc<1>(c, ev.rr, ev.rs, ev.ir, ev.is, yng);
        else sph_solver_nc<0>(c, ev.rr, ev.rs, ev.ir, ev.is, yng);
        for (int b = 0; b < 4; b++) {                  // yspec.f90:367-374
            ysph[0][b] = yng[0][b];
            ysph[1][b] = yng[1][b];
            ysph[2][b] = mk(0.0);
        }
    }
    // the source vectors depend on none of the solve's state: formed after
    // it, they share no stack with the solver's minors
    mcplx svs[5][6];
    source_vector_sph(c, ev.is, ev.rs, ev.mm, svs);
    double zeta = (double)sqrtf((float)(l * (l + 1)));   // yspec.f90:255 (FP32)
    if (ev.pot) {
        // the potential perturbation at the receiver (the third solution
        // component, zero without self-gravitation) in the output type of
        // the event, combined with the source vectors as uu
        if (ev.out != 0) {
            const cd f = out_factor(ev.out, w);
            for (int b = 0; b < 4; b++) ysph[2][b] = f * ysph[2][b];
        }
        for (int q = 0; q < 5; q++) {
            uu[q] = (ysph[2][0] * svs[q][0] + ysph[2][1] * svs[q][1] + ysph[2][2] * svs[q][3] +
                     ysph[2][3] * svs[q][4]) / ev.rr;
            vv[q] = mk(0.0);
        }
        return;
    }
    if (ev.out == 1) {
        cd f = imul(w);
        for (int b = 0; b < 4; b++)
            for (int a = 0; a < 3; a++) ysph[a][b] = f * ysph[a][b];
    } else if (ev.out == 2) {
        cd mw2 = -(w * w);
        if (ev.cor == 0) {
            for (int b = 0; b < 4; b++)
                for (int a = 0; a < 3; a++) ysph[a][b] = mw2 * ysph[a][b];
        } else {                                       // yspec.f90:388-391
            mreal gr = grav_at_receiver(c, ev);
            for (int b = 0; b < 4; b++) {
                mcplx c1 = (-((double)(l + 1) * ysph[2][b] + (2.0 * gr) * ysph[0][b])) / ev.rr;
                mcplx c2 = (zeta * (ysph[2][b] + gr * ysph[0][b])) / ev.rr;
                ysph[0][b] = mw2 * ysph[0][b] + c1;
                ysph[1][b] = mw2 * ysph[1][b] + c2;
            }
        }
    }
    double zr = zeta * ev.rr;
    for (int q = 0; q < 5; q++) {                      // yspec.f90:396-400
        uu[q] = (ysph[0][0] * svs[q][0] + ysph[0][1] * svs[q][1] + ysph[0][2] * svs[q][3] +
                 ysph[0][3] * svs[q][4]) / ev.rr;
        vv[q] = (ysph[1][0] * svs[q][0] + ysph[1][1] * svs[q][1] + ysph[1][2] * svs[q][3] +
                 ysph[1][3] * svs[q][4]) / zr;
    }
}

}  // inline namespace
}  // namespace ysg
#endif  // YSG_SOLVERS_BODY
