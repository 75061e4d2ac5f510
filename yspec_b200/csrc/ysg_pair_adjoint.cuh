// ysg_pair_adjoint.cuh -- reverse sweep of one (omega, l) solve.
//
// The adjoint of pair_radial / pair_toroidal / pair_spheroidal
// (ysg_solvers.cuh) with the source and the receiver in the mantle, the
// receiver above or below the source, with a solid or a fluid inner core
// and with or without an ocean, for every gravity setting (rad_solver_wg /
// rad_solver_ng, tor_solver, sph_solver_g / sph_solver_fic and their
// Cowling and no-gravity forms on both branches, module_solver.f90:25-142,
// :335-561, :640-1740): given the adjoints of the pair's uu / vv /
// ww coefficients, it adds the pair's contribution to dL/dc[i][p][k] (the
// power-form spline segments, see ysg_adjoint.cuh).  No reference
// counterpart: the reference has no derivatives.
//
// Pieces:
//   - the Cash-Karp integrations: yint_log / yint_rev / yint_adj
//     (ysg_adjoint.cuh), every step logged, the minor chain as it runs and
//     the other legs replayed from their stored starts when their adjoint is
//     needed;
//   - the minor algebra (b_solid_start, sph_ysol, the secular determinant,
//     the solid / fluid transforms) is linear in each argument and free of
//     the model: its transposes are formed by applying the forward functions
//     to unit vectors;
//   - the start vectors and the source vectors depend on the thirteen model
//     values at one radius: their derivatives come from the tangent-linear
//     form of the same functions, once per parameter, along "unit" model
//     directions (every knot value of parameter p moved by one, which moves
//     the spline value at every radius by one);
//   - grav(ir), the knot value of the potential / tilt correction, is the c0
//     coefficient of segment ir.
#pragma once
#include "ysg_adjoint.cuh"
#include "ysg_solvers.cuh"

// the tangent-linear form of the same headers (namespace ysg::v_tangent);
// this file's own code goes to the form included first (v_local, or v_loop
// with YSG_LOOPED_STEP), named ysg::primal
#pragma push_macro("YSG_VARIANT")
#pragma push_macro("YSG_TANGENT")
#undef YSG_TANGENT
#define YSG_TANGENT 1
#include "ysg_solvers.cuh"
#pragma pop_macro("YSG_TANGENT")
#pragma pop_macro("YSG_VARIANT")

namespace ysg {
namespace primal = YSG_VARIANT;
inline namespace YSG_VARIANT {

__device__ inline void tangent_ctx(const Ctx& c, const UnitDirs& u, int p, v_tangent::Ctx& t)
{
    t.kn = c.kn;
    t.mh = c.mh;
    t.ll = c.ll;
    t.llp1 = c.llp1;
    t.il = c.il;
    for (int q = 0; q < NSYS; q++) t.nst[q] = 0;
    t.sg = c.sg;
    t.kb = nullptr;
    t.dkn = u.kn[p];
    t.dsg = u.sg[p];
    t.zeta = c.zeta;
    t.zeta2 = c.zeta2;
    t.zeta2m2 = c.zeta2m2;
    t.szeta2m2 = c.szeta2m2;
    t.nu = c.nu;
    t.dr = c.dr;
    t.ats = c.ats;
    t.pib = c.pib;
    t.omega = c.omega;
    t.omega2 = c.omega2;
    t.omegai = c.omegai;
    t.omegai2 = c.omegai2;
    t.lno = c.lno;
}

// vb_p += Re(sum_k yb_k dy_k / dv_p) for the start vectors at (i1, rt) and
// the moments of the result go to G.  WHICH: 0 toroidal (2), 1 solid minor
// (14), 2 fluid minor (5), 3 radial with gravity (2), 4 solid minor without
// self-gravitation (5), 5 fluid start without it (2), 6 radial without
// gravity (2).
template <int WHICH>
__device__ __noinline__ void start_adj(const Ctx& c, const UnitDirs& u, int i1, double rt, const cd* yb, SegGrad& G)
{
    constexpr int N = WHICH == 1 ? 14 : ((WHICH == 2 || WHICH == 4) ? 5 : 2);
    double vb[NPARAM];
    for (int p = 0; p < NPARAM; p++) {
        v_tangent::Ctx t;
        tangent_ctx(c, u, p, t);
        v_tangent::mcplx y[N];
        if (WHICH == 0) v_tangent::tor_ystart(t, i1, rt, y);
        else if (WHICH == 1) v_tangent::sph_minor_solid_start(t, i1, rt, y);
        else if (WHICH == 2) v_tangent::sph_minor_fluid_start(t, i1, rt, y);
        else if (WHICH == 3) v_tangent::rad_ystart<true>(t, i1, rt, y);
        else if (WHICH == 4) v_tangent::sph_minor_solid_start_ng(t, i1, rt, y);
        else if (WHICH == 5) v_tangent::sph_fluid_start_ng(t, i1, rt, y);
        else v_tangent::rad_ystart<false>(t, i1, rt, y);
        double s = 0.0;
        for (int k = 0; k < N; k++) s += re(yb[k] * y[k].d);
        vb[p] = s;
    }
    G.add(i1, rt - c.kn[i1].r, vb);
}

// Source vectors at (is, rs): svtb (5 x 2) and svsb (5 x 6) are the
// adjoints of the toroidal and spheroidal source vectors (either may be
// null).
__device__ __noinline__ void source_adj(const Ctx& c, const UnitDirs& u, int is, double rs, const double* mm,
                                  const cd (*svtb)[2], const cd (*svsb)[6], SegGrad& G)
{
    double vb[NPARAM];
    for (int p = 0; p < NPARAM; p++) {
        v_tangent::Ctx t;
        tangent_ctx(c, u, p, t);
        double s = 0.0;
        if (svtb) {
            v_tangent::mcplx svt[5][2];
            v_tangent::source_vector_tor(t, is, rs, mm, svt);
            for (int q = 0; q < 5; q++)
                for (int b = 0; b < 2; b++) s += re(svtb[q][b] * svt[q][b].d);
        }
        if (svsb) {
            v_tangent::mcplx svs[5][6];
            v_tangent::source_vector_sph(t, is, rs, mm, svs);
            for (int q = 0; q < 5; q++)
                for (int b = 0; b < 6; b++) s += re(svsb[q][b] * svs[q][b].d);
        }
        vb[p] = s;
    }
    G.add(is, rs - c.kn[is].r, vb);
}

// Radial source vector at (is, rs) (module_solver.f90:566-627): s0b holds
// the adjoints of its two components.
__device__ __noinline__ void source_rad_adj(const Ctx& c, const UnitDirs& u, int is, double rs, const double* mm,
                                      const cd* s0b, SegGrad& G)
{
    double vb[NPARAM];
    for (int p = 0; p < NPARAM; p++) {
        v_tangent::Ctx t;
        tangent_ctx(c, u, p, t);
        v_tangent::mcplx s0[2];
        v_tangent::source_vector_rad(t, is, rs, mm, s0);
        vb[p] = re(s0b[0] * s0[0].d) + re(s0b[1] * s0[1].d);
    }
    G.add(is, rs - c.kn[is].r, vb);
}

// ---------------------------------------------------------------------------
// Transposes of the minor algebra (module_int.f90:1563-1837), through the
// forward functions applied to unit vectors.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void unit(cd* e, int n, int j)
{
    for (int k = 0; k < n; k++) e[k] = mk(0.0);
    e[j] = mk(1.0);
}

// y = sph_ysol(m, b): mb += dy/dm^T yb, bb += dy/db^T yb
__device__ inline void ysol_adj(const cd* m, const cd* b, const cd* yb, cd* mb, cd* bb)
{
    cd e[14], y[6];
    for (int j = 0; j < 14; j++) {
        unit(e, 14, j);
        sph_ysol(e, b, y);
        cd s = mk(0.0);
        for (int k = 0; k < 6; k++) s = s + yb[k] * y[k];
        mb[j] = mb[j] + s;
        sph_ysol(m, e, y);
        s = mk(0.0);
        for (int k = 0; k < 6; k++) s = s + yb[k] * y[k];
        bb[j] = bb[j] + s;
    }
}

// d = delta_solid(a, b)
__device__ inline void delta_adj(const cd* a, const cd* b, cd db, cd* ab, cd* bb)
{
    cd e[14];
    for (int j = 0; j < 14; j++) {
        unit(e, 14, j);
        ab[j] = ab[j] + db * delta_solid(e, b);
        bb[j] = bb[j] + db * delta_solid(a, e);
    }
}

// b = b_solid_start(m, s) for a fixed jump s: mb += (db/dm)^T bb
__device__ inline void bstart_adj(const cd* s, const cd* bb, cd* mb)
{
    cd e[14], b[14];
    for (int j = 0; j < 14; j++) {
        unit(e, 14, j);
        b_solid_start(e, s, b);
        cd t = mk(0.0);
        for (int k = 0; k < 14; k++) t = t + bb[k] * b[k];
        mb[j] = mb[j] + t;
    }
}

// mf = s2f(ms): msb += s2f^T mfb;  ms = f2s(mf): mfb += f2s^T msb
__device__ inline void s2f_adj(const cd* mfb, cd* msb)
{
    cd e[14], f[5];
    for (int j = 0; j < 14; j++) {
        unit(e, 14, j);
        s2f(e, f);
        cd t = mk(0.0);
        for (int k = 0; k < 5; k++) t = t + mfb[k] * f[k];
        msb[j] = msb[j] + t;
    }
}
__device__ inline void f2s_adj(const cd* msb, cd* mfb)
{
    cd e[5], m[14];
    for (int j = 0; j < 5; j++) {
        unit(e, 5, j);
        f2s(e, m);
        cd t = mk(0.0);
        for (int k = 0; k < 14; k++) t = t + msb[k] * m[k];
        mfb[j] = mfb[j] + t;
    }
}

// The same for the minor algebra without self-gravitation (the _ngcow
// forms: 5 solid minors, 2 fluid minors, 4-component b-vectors).
__device__ inline void ysol_ngcow_adj(const cd* m, const cd* b, const cd* yb, cd* mb, cd* bb)
{
    cd e[5], y[4];
    for (int j = 0; j < 5; j++) {
        unit(e, 5, j);
        sph_ysol_ngcow(e, b, y);
        cd s = mk(0.0);
        for (int k = 0; k < 4; k++) s = s + yb[k] * y[k];
        mb[j] = mb[j] + s;
    }
    for (int j = 0; j < 4; j++) {
        unit(e, 4, j);
        sph_ysol_ngcow(m, e, y);
        cd s = mk(0.0);
        for (int k = 0; k < 4; k++) s = s + yb[k] * y[k];
        bb[j] = bb[j] + s;
    }
}
__device__ inline void delta_ngcow_adj(const cd* a, const cd* b, cd db, cd* ab, cd* bb)
{
    cd e[5];
    for (int j = 0; j < 5; j++) {
        unit(e, 5, j);
        ab[j] = ab[j] + db * delta_solid_ngcow(e, b);
        bb[j] = bb[j] + db * delta_solid_ngcow(a, e);
    }
}
__device__ inline void bstart_ngcow_adj(const cd* s, const cd* bb, cd* mb)
{
    cd e[5], b[4];
    for (int j = 0; j < 5; j++) {
        unit(e, 5, j);
        b_solid_start_ngcow(e, s, b);
        cd t = mk(0.0);
        for (int k = 0; k < 4; k++) t = t + bb[k] * b[k];
        mb[j] = mb[j] + t;
    }
}
__device__ inline void s2f_ngcow_adj(const cd* mfb, cd* msb)
{
    cd e[5], f[2];
    for (int j = 0; j < 5; j++) {
        unit(e, 5, j);
        s2f_ngcow(e, f);
        msb[j] = msb[j] + mfb[0] * f[0] + mfb[1] * f[1];
    }
}
__device__ inline void f2s_ngcow_adj(const cd* msb, cd* mfb)
{
    cd e[2], m[5];
    for (int j = 0; j < 2; j++) {
        unit(e, 2, j);
        f2s_ngcow(e, m);
        cd t = mk(0.0);
        for (int k = 0; k < 5; k++) t = t + msb[k] * m[k];
        mfb[j] = mfb[j] + t;
    }
}

// ---------------------------------------------------------------------------
// tor_solver (module_solver.f90:25-142), both branches
// ---------------------------------------------------------------------------
// The forward solve again, keeping what the reverse sweep needs, its output
// in yout; yb is the adjoint of yout.  The chain from the start level (to
// the source, or to a receiver below it) is logged as it runs and reversed
// last; the other legs are replayed when reversed.  Returns false if a step
// log overflowed.
__device__ inline bool tor_solver_adj(Ctx& c, const UnitDirs& u, double rr, double rs, int ir, int is,
                                      const cd yb_out[2][2], cd yout[2][2], StepLog& L, StepLog& CL, SegGrad& G)
{
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    int scale1 = 0, scale2 = 0, scale3 = 0;
    cd y1[2], y2[2] = {mk(1.0), mk(0.0)}, y3[2];
    const bool up = rr >= rs;
    const int it = up ? is : ir;
    int i1 = tor_start_level(c, c.ll, c.omega.x, it);
    if (i1 == it && i1 > mh->noc + 1) i1 = i1 - 1;
    const double rt = kn[i1].r;
    const bool cmb_start = i1 == mh->noc + 1;
    if (cmb_start) { y1[0] = mk(1.0); y1[1] = mk(0.0); }
    else tor_ystart(c, i1, rt, y1);
    int n1 = 0;
    if (!yint_log<TorT>(c, i1, it, rt, up ? rs : rr, y1, &scale1, CL, 0, &n1)) return false;
    // the surface solution, from the solid surface down to the receiver
    // (receiver above) or to the source (receiver below)
    const double rbot = up ? rr : rs;
    const int ibot = up ? ir : is;
    const bool down2 = rbot != kn[mh->nsl].r;
    if (down2) yint<TorSys>(c, mh->nsl - 1, ibot, kn[mh->nsl].r, rbot, y2, &scale2);
    // y3 continues the source-side solution from the source to the receiver
    const cd* y3s = up ? y1 : y2;
    y3[0] = y3s[0];
    y3[1] = y3s[1];
    const cd y3start[2] = {y3s[0], y3s[1]};
    if (rr != rs) yint<TorSys>(c, is, ir, rs, rr, y3, &scale3);
    // D = P[1] Q[0] - P[0] Q[1]: (P, Q) = (y2, y3) above, (y3, y1) below;
    // b from the source-side solution (y1 above, y2 below), the receiver's
    // solution dy = delta (y2 above, y1 below)
    const cd* P = up ? y2 : y3;
    const cd* Q = up ? y3 : y1;
    const cd D = P[1] * Q[0] - P[0] * Q[1];
    const cd delta = 1.0 / D;
    const cd* Bs = up ? y1 : y2;
    const cd* R = up ? y2 : y1;
    const cd bv[2] = {Bs[1], -Bs[0]};
    const cd dy[2] = {delta * R[0], delta * R[1]};
    const double F = huge_pow(scale3);
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) yout[a][b] = F * (-(dy[a] * bv[b]));
    // reverse: yout[a][b] = -F delta R[a] bv[b]
    cd dyb[2] = {mk(0.0), mk(0.0)}, bvb[2] = {mk(0.0), mk(0.0)};
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) {
            const cd g = F * yb_out[a][b];
            dyb[a] = dyb[a] - g * bv[b];
            bvb[b] = bvb[b] - g * dy[a];
        }
    cd y1b[2] = {mk(0.0), mk(0.0)}, y2b[2] = {mk(0.0), mk(0.0)}, y3b[2] = {mk(0.0), mk(0.0)};
    cd* Bsb = up ? y1b : y2b;
    cd* Rb = up ? y2b : y1b;
    cd* Pb = up ? y2b : y3b;
    cd* Qb = up ? y3b : y1b;
    Bsb[1] = Bsb[1] + bvb[0];
    Bsb[0] = Bsb[0] - bvb[1];
    const cd deltab = dyb[0] * R[0] + dyb[1] * R[1];
    Rb[0] = Rb[0] + delta * dyb[0];
    Rb[1] = Rb[1] + delta * dyb[1];
    const cd Db = -(deltab * (delta * delta));
    Pb[1] = Pb[1] + Db * Q[0];
    Pb[0] = Pb[0] - Db * Q[1];
    Qb[0] = Qb[0] + Db * P[1];
    Qb[1] = Qb[1] - Db * P[0];
    // y3 from its start at the source
    if (rr != rs && !yint_adj<TorT>(c, is, ir, rs, rr, y3start, y3b, true, L, G)) return false;
    cd* y3sb = up ? y1b : y2b;
    y3sb[0] = y3sb[0] + y3b[0];
    y3sb[1] = y3sb[1] + y3b[1];
    // the surface solution starts from a fixed vector: only its model gradient
    const cd e2[2] = {mk(1.0), mk(0.0)};
    if (down2 && !yint_adj<TorT>(c, mh->nsl - 1, ibot, kn[mh->nsl].r, rbot, e2, y2b, true, L, G)) return false;
    yint_rev<TorT>(c, CL, 0, n1, y1b, G);
    if (!cmb_start) start_adj<0>(c, u, i1, rt, y1b, G);
    return true;
}

// ---------------------------------------------------------------------------
// sph_solver_g and sph_solver_fic (module_solver.f90:640-823, :1203-1382),
// both branches, with or without an ocean: yb_out (6 x 4) is the adjoint
// of yout.
// ---------------------------------------------------------------------------
__device__ inline bool sph_solver_g_adj(Ctx& c, const UnitDirs& u, double rr, double rs, int ir, int is,
                                        const cd yb_out[6][4], cd yout[6][4], StepLog& L, StepLog& CL,
                                        SegGrad& G)
{
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    int scale1 = 0, scale2 = 0, scale3 = 0;
    const bool up = rr >= rs;
    const int it = up ? is : ir;
    const double rtop = up ? rs : rr;
    int i1 = sph_start_level(c, c.ll, c.omega.x, it);
    double rt = kn[i1].r;
    if (i1 == 1 && (up || mh->fic)) rt = fmin(0.1 * c.dr, 0.1 * kn[2].r);
    if (i1 >= it) { i1 = it - 1; rt = kn[i1].r; }
    // The chain from the start level to the source (receiver above) or to
    // the receiver (receiver below); branch 0: solid inner core start, 1:
    // fluid start (outer core, or a fluid inner core, which starts from the
    // fluid minor there as the outer core does), 2: mantle start.  Its legs
    // (inner core, outer core, mantle) are logged as they run, one after
    // the other in the chain log, and reversed in the opposite order at the
    // end; the other integrations are replayed in the scratch log when
    // reversed.
    const int branch = (i1 <= mh->nic && !mh->fic) ? 0 : (i1 <= mh->noc ? 1 : 2);
    cd st[14], ms1[14], mf[5];
    int nic_s = 0, noc_s = 0, nm_s = 0;                          // steps of the three legs
    if (branch == 0) {
        sph_minor_solid_start(c, i1, rt, st);
        for (int k = 0; k < 14; k++) ms1[k] = st[k];
        if (!yint_log<MinorSolidGT>(c, i1, mh->nic, rt, kn[mh->nic].r, ms1, &scale1, CL, 0, &nic_s)) return false;
        s2f(ms1, mf);
        if (!yint_log<MinorFluidGT>(c, mh->nic + 1, mh->noc, kn[mh->nic].r, kn[mh->noc].r, mf, &scale1, CL, nic_s,
                                    &noc_s))
            return false;
        f2s(mf, ms1);
    } else if (branch == 1) {
        sph_minor_fluid_start(c, i1, rt, mf);
        if (!yint_log<MinorFluidGT>(c, i1, mh->noc, rt, kn[mh->noc].r, mf, &scale1, CL, 0, &noc_s)) return false;
        f2s(mf, ms1);
    } else {
        sph_minor_solid_start(c, i1, rt, st);
        for (int k = 0; k < 14; k++) ms1[k] = st[k];
    }
    const int mi1 = branch == 2 ? i1 : mh->noc + 1;
    const double mr1 = branch == 2 ? rt : kn[mh->noc + 1].r;
    const int moff = nic_s + noc_s;
    if (!yint_log<MinorSolidGT>(c, mi1, it, mr1, rtop, ms1, &scale1, CL, moff, &nm_s)) return false;
    // ms3 continues the chain between the receiver and the source
    cd ms3[14], ms2[14];
    for (int k = 0; k < 14; k++) ms3[k] = ms1[k];
    const bool leg3 = up ? rr > rs : rs > rr;
    const int l3a = up ? is : ir, l3b = up ? ir : is;
    const double r3a = up ? rs : rr, r3b = up ? rr : rs;
    if (leg3) yint<MinorSolidG>(c, l3a, l3b, r3a, r3b, ms3, &scale3);
    // the solution from the surface down to the receiver (receiver above) or
    // to the source (below): through an ocean first (a fluid minor from the
    // surface to its floor, then the solid minor from the floor), else the
    // solid minor from the surface
    const int ibot = up ? ir : is;
    const double rbot = up ? rr : rs;
    cd e1[14], mo[5], ms2s[14];
    unit(e1, 14, 0);
    for (int k = 0; k < 14; k++) ms2[k] = e1[k];
    unit(mo, 5, 0);
    if (mh->ocean) {
        cd mf2[5];
        for (int k = 0; k < 5; k++) mf2[k] = mo[k];
        yint<MinorFluidG>(c, mh->nknot - 1, mh->nsl + 1, kn[mh->nknot].r, kn[mh->nsl + 1].r, mf2, &scale2);
        f2s(mf2, ms2);
    }
    const int s2i1 = mh->ocean ? mh->nsl : (up ? mh->nknot - 1 : mh->nknot);
    const double s2r1 = mh->ocean ? kn[mh->nsl].r : kn[mh->nknot].r;
    for (int k = 0; k < 14; k++) ms2s[k] = ms2[k];
    yint<MinorSolidG>(c, s2i1, ibot, s2r1, rbot, ms2, &scale2);
    const cd delta = delta_solid(ms3, ms2);
    const int jump[4] = {0, 1, 3, 4};
    cd ms1b[14], ms2b[14], ms3b[14];
    for (int k = 0; k < 14; k++) ms1b[k] = ms2b[k] = ms3b[k] = mk(0.0);
    cd deltab = mk(0.0);
    // the b-vector of each jump from the source to the receiver
    cd* const mst = up ? ms1 : ms2;                 // the minors it starts from
    cd* const mstb = up ? ms1b : ms2b;
    cd* const mso = up ? ms2 : ms1;                 // the minors it is read with
    cd* const msob = up ? ms2b : ms1b;
    for (int i = 0; i < 4; i++) {
        cd s[6];
        unit(s, 6, jump[i]);
        int scale4 = 0;
        cd b[14], b0[14], ys[6];
        b_solid_start(mst, s, b0);
        for (int k = 0; k < 14; k++) b[k] = up ? b0[k] : (-b0[k]) / delta;
        int nb = 0;
        if (!yint_log<BvecSolidGT>(c, is, ir, rs, rr, b, &scale4, L, 0, &nb)) return false;
        sph_ysol(mso, b, ys);
        const double F = huge_pow(scale3 - scale4);
        cd ysb[6];
        for (int k = 0; k < 6; k++) {
            const cd yk = F * yb_out[k][i];
            if (up) {
                // yout[k][i] = (-ys[k] / delta) F
                yout[k][i] = F * (-(ys[k] / delta));
                ysb[k] = -(yk / delta);
                deltab = deltab + yk * (ys[k] / (delta * delta));
            } else {
                // yout[k][i] = ys[k] F, the start divided by -delta
                yout[k][i] = F * ys[k];
                ysb[k] = yk;
            }
        }
        cd bb[14];
        for (int k = 0; k < 14; k++) bb[k] = mk(0.0);
        ysol_adj(mso, b, ysb, msob, bb);
        yint_rev<BvecSolidGT>(c, L, 0, nb, bb, G);
        if (!up) {
            // b = -b0 / delta
            for (int k = 0; k < 14; k++) {
                deltab = deltab + bb[k] * (b0[k] / (delta * delta));
                bb[k] = -(bb[k] / delta);
            }
        }
        bstart_adj(s, bb, mstb);
    }
    delta_adj(ms3, ms2, deltab, ms3b, ms2b);
    if (!yint_adj<MinorSolidGT>(c, s2i1, ibot, s2r1, rbot, ms2s, ms2b, true, L, G)) return false;
    if (mh->ocean) {
        // back through the ocean: the fluid minor starts from a fixed vector
        cd mf2b[5];
        for (int k = 0; k < 5; k++) mf2b[k] = mk(0.0);
        f2s_adj(ms2b, mf2b);
        if (!yint_adj<MinorFluidGT>(c, mh->nknot - 1, mh->nsl + 1, kn[mh->nknot].r, kn[mh->nsl + 1].r, mo, mf2b,
                                    true, L, G))
            return false;
    }
    if (leg3 && !yint_adj<MinorSolidGT>(c, l3a, l3b, r3a, r3b, ms1, ms3b, true, L, G)) return false;
    for (int k = 0; k < 14; k++) ms1b[k] = ms1b[k] + ms3b[k];
    // back along the chain to the start level
    yint_rev<MinorSolidGT>(c, CL, moff, nm_s, ms1b, G);
    if (branch == 2) {
        start_adj<1>(c, u, i1, rt, ms1b, G);
        return true;
    }
    cd mfb[5];
    for (int k = 0; k < 5; k++) mfb[k] = mk(0.0);
    f2s_adj(ms1b, mfb);
    yint_rev<MinorFluidGT>(c, CL, nic_s, noc_s, mfb, G);
    if (branch == 1) {
        start_adj<2>(c, u, i1, rt, mfb, G);
        return true;
    }
    cd msb[14];
    for (int k = 0; k < 14; k++) msb[k] = mk(0.0);
    s2f_adj(mfb, msb);
    yint_rev<MinorSolidGT>(c, CL, 0, nic_s, msb, G);
    start_adj<1>(c, u, i1, rt, msb, G);
    return true;
}

// ---------------------------------------------------------------------------
// sph_solver_nc without self-gravitation (KIND 0, module_solver.f90:827-1010)
// and in the Cowling approximation (KIND 1, :1014-1195), with their fluid
// inner core forms (:1386-1740), both branches: the same sweep as
// sph_solver_g_adj on the 5-minor / 2-minor / 4-vector systems.
// ---------------------------------------------------------------------------
template <int KIND>
__device__ inline bool sph_solver_nc_adj(Ctx& c, const UnitDirs& u, double rr, double rs, int ir, int is,
                                         const cd yb_out[4][4], cd yout[4][4], StepLog& L, StepLog& CL,
                                         SegGrad& G)
{
    using SolidT = MinorSolidNCT<KIND>;
    using FluidT = MinorFluidNCT<KIND>;
    using BvecT = BvecSolidNCT<KIND>;
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    int scale1 = 0, scale2 = 0, scale3 = 0;
    const bool up = rr >= rs;
    const int it = up ? is : ir;
    const double rtop = up ? rs : rr;
    int i1 = sph_start_level(c, c.ll, c.omega.x, it);
    double rt = kn[i1].r;
    if (i1 == 1 && (up || mh->fic)) rt = fmin(0.1 * c.dr, 0.1 * kn[2].r);
    if (i1 >= it) { i1 = it - 1; rt = kn[i1].r; }
    // branch 0: solid inner core start, 1: fluid start (outer core, or a
    // fluid inner core), 2: mantle start; the chain's legs in the chain log
    const int branch = (i1 <= mh->nic && !mh->fic) ? 0 : (i1 <= mh->noc ? 1 : 2);
    cd ms1[5], mf[2];
    int nic_s = 0, noc_s = 0, nm_s = 0;
    if (branch == 0) {
        sph_minor_solid_start_ng(c, i1, rt, ms1);
        if (!yint_log<SolidT>(c, i1, mh->nic, rt, kn[mh->nic].r, ms1, &scale1, CL, 0, &nic_s)) return false;
        s2f_ngcow(ms1, mf);
        if (!yint_log<FluidT>(c, mh->nic + 1, mh->noc, kn[mh->nic].r, kn[mh->noc].r, mf, &scale1, CL, nic_s, &noc_s))
            return false;
        f2s_ngcow(mf, ms1);
    } else if (branch == 1) {
        sph_fluid_start_ng(c, i1, rt, mf);
        if (!yint_log<FluidT>(c, i1, mh->noc, rt, kn[mh->noc].r, mf, &scale1, CL, 0, &noc_s)) return false;
        f2s_ngcow(mf, ms1);
    } else {
        sph_minor_solid_start_ng(c, i1, rt, ms1);
    }
    const int mi1 = branch == 2 ? i1 : mh->noc + 1;
    const double mr1 = branch == 2 ? rt : kn[mh->noc + 1].r;
    const int moff = nic_s + noc_s;
    if (!yint_log<SolidT>(c, mi1, it, mr1, rtop, ms1, &scale1, CL, moff, &nm_s)) return false;
    cd ms3[5], ms2[5], ms2s[5], mo[2];
    for (int k = 0; k < 5; k++) ms3[k] = ms1[k];
    const bool leg3 = up ? rr > rs : rs > rr;
    const int l3a = up ? is : ir, l3b = up ? ir : is;
    const double r3a = up ? rs : rr, r3b = up ? rr : rs;
    if (leg3) yint<MinorSolidNC<KIND>>(c, l3a, l3b, r3a, r3b, ms3, &scale3);
    // from the surface down to the receiver (above) or the source (below),
    // through an ocean first
    const int ibot = up ? ir : is;
    const double rbot = up ? rr : rs;
    unit(ms2, 5, 0);
    unit(mo, 2, 0);
    if (mh->ocean) {
        cd mf2[2] = {mo[0], mo[1]};
        yint<MinorFluidNC<KIND>>(c, mh->nknot - 1, mh->nsl + 1, kn[mh->nknot].r, kn[mh->nsl + 1].r, mf2, &scale2);
        f2s_ngcow(mf2, ms2);
    }
    const int s2i1 = mh->ocean ? mh->nsl : mh->nknot;
    const double s2r1 = mh->ocean ? kn[mh->nsl].r : kn[mh->nknot].r;
    for (int k = 0; k < 5; k++) ms2s[k] = ms2[k];
    yint<MinorSolidNC<KIND>>(c, s2i1, ibot, s2r1, rbot, ms2, &scale2);
    const cd delta = delta_solid_ngcow(ms3, ms2);
    cd ms1b[5], ms2b[5], ms3b[5];
    for (int k = 0; k < 5; k++) ms1b[k] = ms2b[k] = ms3b[k] = mk(0.0);
    cd deltab = mk(0.0);
    // the b-vector of each jump starts from the chain's end (receiver
    // above) or from the surface solution divided by -delta (below), and is
    // read at the receiver with the other
    cd* const mst = up ? ms1 : ms2;
    cd* const mstb = up ? ms1b : ms2b;
    cd* const mso = up ? ms2 : ms1;
    cd* const msob = up ? ms2b : ms1b;
    for (int i = 0; i < 4; i++) {
        cd s[4], b[4], b0[4], ys[4];
        unit(s, 4, i);
        b_solid_start_ngcow(mst, s, b0);
        for (int k = 0; k < 4; k++) b[k] = up ? b0[k] : (-b0[k]) / delta;
        int scale4 = 0, nb = 0;
        if (!yint_log<BvecT>(c, is, ir, rs, rr, b, &scale4, L, 0, &nb)) return false;
        sph_ysol_ngcow(mso, b, ys);
        const double F = huge_pow(scale3 - scale4);
        cd ysb[4];
        for (int k = 0; k < 4; k++) {
            const cd yk = F * yb_out[k][i];
            if (up) {
                // yout[k][i] = (ys[k] / delta) huge^(scale3 - scale4)
                yout[k][i] = F * (ys[k] / delta);
                ysb[k] = yk / delta;
                deltab = deltab - yk * (ys[k] / (delta * delta));
            } else {
                yout[k][i] = F * ys[k];
                ysb[k] = yk;
            }
        }
        cd bb[4] = {mk(0.0), mk(0.0), mk(0.0), mk(0.0)};
        ysol_ngcow_adj(mso, b, ysb, msob, bb);
        yint_rev<BvecT>(c, L, 0, nb, bb, G);
        if (!up) {
            for (int k = 0; k < 4; k++) {
                deltab = deltab + bb[k] * (b0[k] / (delta * delta));
                bb[k] = -(bb[k] / delta);
            }
        }
        bstart_ngcow_adj(s, bb, mstb);
    }
    delta_ngcow_adj(ms3, ms2, deltab, ms3b, ms2b);
    if (!yint_adj<SolidT>(c, s2i1, ibot, s2r1, rbot, ms2s, ms2b, true, L, G)) return false;
    if (mh->ocean) {
        cd mf2b[2] = {mk(0.0), mk(0.0)};
        f2s_ngcow_adj(ms2b, mf2b);
        if (!yint_adj<FluidT>(c, mh->nknot - 1, mh->nsl + 1, kn[mh->nknot].r, kn[mh->nsl + 1].r, mo, mf2b, true, L,
                              G))
            return false;
    }
    if (leg3 && !yint_adj<SolidT>(c, l3a, l3b, r3a, r3b, ms1, ms3b, true, L, G)) return false;
    for (int k = 0; k < 5; k++) ms1b[k] = ms1b[k] + ms3b[k];
    yint_rev<SolidT>(c, CL, moff, nm_s, ms1b, G);
    if (branch == 2) {
        start_adj<4>(c, u, i1, rt, ms1b, G);
        return true;
    }
    cd mfb[2] = {mk(0.0), mk(0.0)};
    f2s_ngcow_adj(ms1b, mfb);
    yint_rev<FluidT>(c, CL, nic_s, noc_s, mfb, G);
    if (branch == 1) {
        start_adj<5>(c, u, i1, rt, mfb, G);
        return true;
    }
    cd msb[5] = {mk(0.0), mk(0.0), mk(0.0), mk(0.0), mk(0.0)};
    s2f_ngcow_adj(mfb, msb);
    yint_rev<SolidT>(c, CL, 0, nic_s, msb, G);
    start_adj<4>(c, u, i1, rt, msb, G);
    return true;
}

// Grid of the l = 0 gravity solve (rad_solver_wg): per grid point k its
// radius, interval and the upward and downward solutions there.  Entry e
// of an array sits at e * st, as in StepLog.
struct GridLog {
    cd* y;            // nmax x 4: upward y1[0], y1[1], downward y2[0], y2[1]
    double* r;        // nmax
    int* i;           // nmax
    int nmax;
    int st;
};

// rad_solver_wg (ysg_solvers.cuh, module_solver.f90:446-561) run forward
// with every grid point stored, its result in yout, then reversed: yb holds
// the adjoints of yout.  The grid walk is the forward one, point for point;
// each piece between grid points is replayed from its stored start by
// yint_adj.  Returns false if the grid or a piece exceeds the logs, or the
// receiver is not on the grid.
__device__ inline bool rad_solver_wg_adj(Ctx& c, const UnitDirs& u, double rr, double rs, const cd yb[2][2],
                                         cd yout[2][2], StepLog& L, GridLog& GL, SegGrad& G)
{
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    const double drr = c.dr;
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
    if (ngrid + 1 > GL.nmax || iss < 2 || irr < 2) return false;
    const int st = GL.st;
    auto gy = [&](int k, int s) -> cd& { return GL.y[((size_t)k * 4 + s) * st]; };
    // upward through grid points 2..iss
    cd y1[2], ys[2];
    double rt = 0.0;
    {
        int k = 0, iprev = 0;
        double rprev = 0.0;
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
                    GL.r[(size_t)k * st] = rk;
                    GL.i[(size_t)k * st] = i;
                    if (k == 2) {
                        rt = fmin(0.1 * drr, 0.1 * rk);
                        rad_ystart<true>(c, 1, rt, ys);
                        y1[0] = ys[0]; y1[1] = ys[1];
                        yint<RadSys>(c, 1, i, rt, rk, y1, nullptr);
                    } else if (k > 2) {
                        yint<RadSys>(c, iprev, i, rprev, rk, y1, nullptr);
                    }
                    if (k >= 2) { gy(k, 0) = y1[0]; gy(k, 1) = y1[1]; }
                    iprev = i;
                    rprev = rk;
                }
            }
        }
    }
    // downward from grid point ngrid to iss
    cd y2[2] = {mk(1.0), mk(0.0)};
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
                    GL.r[(size_t)k * st] = rk;
                    GL.i[(size_t)k * st] = i;
                    if (k < ngrid) yint<RadSys>(c, iprev, i, rprev, rk, y2, nullptr);
                    gy(k, 2) = y2[0];
                    gy(k, 3) = y2[1];
                    iprev = i;
                    rprev = rk;
                }
            }
        }
    }
    const bool rec_up = irr <= iss;               // receiver on the upward walk
    const cd yrec[2] = {gy(irr, rec_up ? 0 : 2), gy(irr, rec_up ? 1 : 3)};
    const cd D = y2[1] * y1[0] - y2[0] * y1[1];
    const cd delta = 1.0 / D;
    const cd* Y = rec_up ? y2 : y1;
    const cd bv[2] = {Y[1], -Y[0]};
    const cd dy[2] = {delta * yrec[0], delta * yrec[1]};
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) yout[a][b] = -(dy[a] * bv[b]);
    // reverse: yout[a][b] = -delta yrec[a] bv[b]
    cd dyb[2] = {mk(0.0), mk(0.0)}, bvb[2] = {mk(0.0), mk(0.0)};
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) {
            dyb[a] = dyb[a] - yb[a][b] * bv[b];
            bvb[b] = bvb[b] - yb[a][b] * dy[a];
        }
    const cd deltab = dyb[0] * yrec[0] + dyb[1] * yrec[1];
    const cd yrecb[2] = {dyb[0] * delta, dyb[1] * delta};
    const cd Db = -(deltab * (delta * delta));
    cd y1b[2] = {Db * y2[1], -(Db * y2[0])};
    cd y2b[2] = {-(Db * y1[1]), Db * y1[0]};
    cd* Yb = rec_up ? y2b : y1b;
    Yb[1] = Yb[1] + bvb[0];
    Yb[0] = Yb[0] - bvb[1];
    // downward walk, reversed: y2(k) = piece(k+1 -> k) y2(k+1)
    for (int k = iss; k < ngrid; k++) {
        if (!rec_up && k == irr) {
            y2b[0] = y2b[0] + yrecb[0];
            y2b[1] = y2b[1] + yrecb[1];
        }
        const cd yin[2] = {gy(k + 1, 2), gy(k + 1, 3)};
        if (!yint_adj<RadT>(c, GL.i[(size_t)(k + 1) * st], GL.i[(size_t)k * st], GL.r[(size_t)(k + 1) * st],
                            GL.r[(size_t)k * st], yin, y2b, false, L, G))
            return false;
    }
    // upward walk, reversed: y1(k) = piece(k-1 -> k) y1(k-1), y1(2) from the start
    for (int k = iss; k >= 2; k--) {
        if (rec_up && k == irr) {
            y1b[0] = y1b[0] + yrecb[0];
            y1b[1] = y1b[1] + yrecb[1];
        }
        if (k > 2) {
            const cd yin[2] = {gy(k - 1, 0), gy(k - 1, 1)};
            if (!yint_adj<RadT>(c, GL.i[(size_t)(k - 1) * st], GL.i[(size_t)k * st], GL.r[(size_t)(k - 1) * st],
                                GL.r[(size_t)k * st], yin, y1b, false, L, G))
                return false;
        } else {
            if (!yint_adj<RadT>(c, 1, GL.i[(size_t)k * st], rt, GL.r[(size_t)k * st], ys, y1b, false, L, G))
                return false;
            start_adj<3>(c, u, 1, rt, y1b, G);
        }
    }
    return true;
}

// rad_solver_ng (ysg_solvers.cuh, module_solver.f90:335-441; the radial
// system in its gravity form, rad_derivs_ng), both branches: the forward
// pass (its upward leg from the centre to the source or receiver in the
// chain log), its output in yout, then the reverse sweep from yb.
__device__ inline bool rad_solver_ng_adj(Ctx& c, const UnitDirs& u, double rr, double rs, int ir, int is,
                                         const cd yb[2][2], cd yout[2][2], StepLog& L, StepLog& CL, SegGrad& G)
{
    const ModelHdr* mh = c.mh;
    const Knot* kn = c.kn;
    const bool up = rr >= rs;
    int scale1 = 0, scale2 = 0, scale3 = 0, n1 = 0;
    const double rt = fmin(0.1 * c.dr, 0.1 * kn[2].r);
    cd y1[2], y2[2] = {mk(1.0), mk(0.0)}, y3[2], y2s[2];
    rad_ystart<false>(c, 1, rt, y1);
    // the upward leg ends at the lower of the two points, the downward leg
    // starts at the surface (above) or the top of the solid (below)
    const int ilo = up ? is : ir, ihi = up ? ir : is;
    const double rlo = up ? rs : rr, rhi = up ? rr : rs;
    const int top = up ? mh->nknot : mh->nsl;
    if (!yint_log<RadT>(c, 1, ilo, rt, rlo, y1, &scale1, CL, 0, &n1)) return false;
    const bool leg2 = rhi != kn[top].r, leg3 = rs != rr;
    if (leg2) yint<RadSys>(c, top - 1, ihi, kn[top].r, rhi, y2, &scale2);
    y2s[0] = y2[0];
    y2s[1] = y2[1];
    y3[0] = y2[0];
    y3[1] = y2[1];
    if (leg3) yint<RadSys>(c, ihi, ilo, rhi, rlo, y3, &scale3);
    const cd D = y3[1] * y1[0] - y3[0] * y1[1];
    const bool degenerate = cabs(D) < 1.0e-100;
    const cd delta = degenerate ? mk(0.0) : 1.0 / D;
    // ya forms b, yr is read at the receiver
    const cd* ya = up ? y1 : y2;
    const cd* yr = up ? y2 : y1;
    const cd bv[2] = {ya[1], -ya[0]};
    const cd dy[2] = {delta * yr[0], delta * yr[1]};
    // the receiver-below branch undoes only a positive scale3
    // (module_solver.f90:433-437)
    const double F = (up ? scale3 != 0 : scale3 > 0) ? huge_pow(scale3) : 1.0;
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) yout[a][b] = F * (-(dy[a] * bv[b]));
    // reverse: yout[a][b] = -F delta yr[a] bv[b]
    cd dyb[2] = {mk(0.0), mk(0.0)}, bvb[2] = {mk(0.0), mk(0.0)};
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++) {
            const cd g = F * yb[a][b];
            dyb[a] = dyb[a] - g * bv[b];
            bvb[b] = bvb[b] - g * dy[a];
        }
    const cd yab[2] = {-bvb[1], bvb[0]};
    const cd deltab = dyb[0] * yr[0] + dyb[1] * yr[1];
    const cd yrb[2] = {delta * dyb[0], delta * dyb[1]};
    cd y1b[2], y2b[2];
    for (int k = 0; k < 2; k++) {
        y1b[k] = up ? yab[k] : yrb[k];
        y2b[k] = up ? yrb[k] : yab[k];
    }
    cd y3b[2] = {mk(0.0), mk(0.0)};
    if (!degenerate) {
        const cd Db = -(deltab * (delta * delta));
        y3b[0] = -(Db * y1[1]);
        y3b[1] = Db * y1[0];
        y1b[0] = y1b[0] + Db * y3[1];
        y1b[1] = y1b[1] - Db * y3[0];
    }
    if (leg3 && !yint_adj<RadT>(c, ihi, ilo, rhi, rlo, y2s, y3b, true, L, G)) return false;
    y2b[0] = y2b[0] + y3b[0];
    y2b[1] = y2b[1] + y3b[1];
    const cd e[2] = {mk(1.0), mk(0.0)};
    if (leg2 && !yint_adj<RadT>(c, top - 1, ihi, kn[top].r, rhi, e, y2b, true, L, G)) return false;
    yint_rev<RadT>(c, CL, 0, n1, y1b, G);
    start_adj<6>(c, u, 1, rt, y1b, G);
    return true;
}

// ---------------------------------------------------------------------------
// The per-pair epilogues of yspec.f90:301-316 and :344-400.
// ---------------------------------------------------------------------------
// coefb: adjoints of the 15 coefficients of pair (l = 0, j); only uu(3)
// is formed by the radial solve (yspec.f90:263-293).
__device__ inline bool pair_radial_adj(Ctx& c, const UnitDirs& u, const EventDev& ev, int j, const cd* coefb,
                                       StepLog& L, StepLog& CL, GridLog& GL, SegGrad& G)
{
    const cd w = omega_of(ev, j);
    set_l(c, 0);
    set_omega(c, w);
    cd sr0[2], yrad[2][2];
    source_vector_rad(c, ev.is, ev.rs, ev.mm, sr0);
    alpha_steps(c);
    // u3 = f (sr0[0] yrad[0][0] + sr0[1] yrad[0][1]) / rr
    cd g = coefb[2];
    if (ev.out != 0) g = out_factor(ev.out, w) * g;
    g = g / ev.rr;
    const cd yb[2][2] = {{g * sr0[0], g * sr0[1]}, {mk(0.0), mk(0.0)}};
    if (ev.grav == 0) {
        if (!rad_solver_ng_adj(c, u, ev.rr, ev.rs, ev.ir, ev.is, yb, yrad, L, CL, G)) return false;
    } else if (!rad_solver_wg_adj(c, u, ev.rr, ev.rs, yb, yrad, L, GL, G)) {
        return false;
    }
    const cd s0b[2] = {g * yrad[0][0], g * yrad[0][1]};
    source_rad_adj(c, u, ev.is, ev.rs, ev.mm, s0b, G);
    return true;
}

// wwb: adjoints of ww(1:5) of pair (l >= 2, j).  The adjoints of the
// solver's output need only the source vectors, so the solver's reverse
// sweep runs first and its own forward pass supplies the output that the
// source vectors' adjoints need.
__device__ inline bool pair_toroidal_adj(Ctx& c, const UnitDirs& u, const EventDev& ev, int l, int j,
                                         const cd* wwb, StepLog& L, StepLog& CL, SegGrad& G)
{
    const cd w = omega_of(ev, j);
    set_l(c, l);
    set_omega(c, w);
    cd svt[5][2], ytor[2][2];
    source_vector_tor(c, ev.is, ev.rs, ev.mm, svt);
    const cd f = out_factor(ev.out, w);
    const double zeta = (double)sqrtf((float)(l * (l + 1)));
    const double zr = zeta * ev.rr;
    // ww[q] = (svt[q][0] ytor'[0][0] + svt[q][1] ytor'[0][1]) / zr, ytor' = f ytor
    cd yb[2][2] = {{mk(0.0), mk(0.0)}, {mk(0.0), mk(0.0)}};
    for (int q = 0; q < 5; q++) {
        const cd g = wwb[q] / zr;
        yb[0][0] = yb[0][0] + g * svt[q][0];
        yb[0][1] = yb[0][1] + g * svt[q][1];
    }
    if (ev.out != 0)
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) yb[a][b] = f * yb[a][b];
    if (!tor_solver_adj(c, u, ev.rr, ev.rs, ev.ir, ev.is, yb, ytor, L, CL, G)) return false;
    if (ev.out != 0)
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) ytor[a][b] = f * ytor[a][b];
    cd svtb[5][2];
    for (int q = 0; q < 5; q++) {
        const cd g = wwb[q] / zr;
        svtb[q][0] = g * ytor[0][0];
        svtb[q][1] = g * ytor[0][1];
    }
    source_adj(c, u, ev.is, ev.rs, ev.mm, svtb, nullptr, G);
    return true;
}

// uub, vvb: adjoints of uu(1:5), vv(1:5) of pair (l >= 1, j); the same
// order as the toroidal part.
__device__ inline bool pair_spheroidal_adj(Ctx& c, const UnitDirs& u, const EventDev& ev, int l, int j,
                                           const cd* uub, const cd* vvb, StepLog& L, StepLog& CL, SegGrad& G)
{
    const cd w = omega_of(ev, j);
    set_l(c, l);
    set_omega(c, w);
    alpha_steps(c);
    cd svs[5][6], ysph[6][4];
    source_vector_sph(c, ev.is, ev.rs, ev.mm, svs);
    const double zeta = (double)sqrtf((float)(l * (l + 1)));
    const cd mw2 = -(w * w);
    const double gr = ev.grav_ir;
    const double zr = zeta * ev.rr;
    const int col[4] = {0, 1, 3, 4};
    // uu[q] = sum_b ysph'[0][b] svs[q][col b] / rr;  vv[q] = sum_b ysph'[1][b] svs[q][col b] / zr,
    // ysph' the solver output after the output scaling and corrections
    cd yb[6][4], ybo[2][4];
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 4; b++) yb[a][b] = mk(0.0);
    for (int q = 0; q < 5; q++) {
        const cd gu = uub[q] / ev.rr, gv = vvb[q] / zr;
        for (int b = 0; b < 4; b++) {
            yb[0][b] = yb[0][b] + gu * svs[q][col[b]];
            yb[1][b] = yb[1][b] + gv * svs[q][col[b]];
        }
    }
    for (int b = 0; b < 4; b++) {
        ybo[0][b] = yb[0][b];
        ybo[1][b] = yb[1][b];
    }
    // output scaling and the potential / tilt correction (yspec.f90:376-391)
    if (ev.out == 1) {
        const cd f = imul(w);
        for (int b = 0; b < 4; b++)
            for (int a = 0; a < 3; a++) yb[a][b] = f * yb[a][b];
    } else if (ev.out == 2) {
        if (ev.cor == 0) {
            for (int b = 0; b < 4; b++)
                for (int a = 0; a < 3; a++) yb[a][b] = mw2 * yb[a][b];
        } else {
            for (int b = 0; b < 4; b++) {
                const cd a0 = yb[0][b], a1 = yb[1][b];
                // y0' = mw2 y0 - ((l+1) y2 + 2 g y0) / rr;  y1' = mw2 y1 + zeta (y2 + g y0) / rr
                yb[0][b] = a0 * (mw2 - (2.0 * gr) / ev.rr) + a1 * (zeta * gr / ev.rr);
                yb[1][b] = a1 * mw2;
                yb[2][b] = yb[2][b] + a0 * (-(double)(l + 1) / ev.rr) + a1 * (zeta / ev.rr);
            }
        }
    }
    if (ev.grav == 2) {
        if (!sph_solver_g_adj(c, u, ev.rr, ev.rs, ev.ir, ev.is, yb, ysph, L, CL, G)) return false;
    } else {
        // the 4-vector solution (U, V, R, S): its U and V rows are the
        // outputs; the potential is zero (yspec.f90:367-374)
        cd ybn[4][4], yng[4][4];
        for (int b = 0; b < 4; b++) {
            ybn[0][b] = yb[0][b];
            ybn[1][b] = yb[1][b];
            ybn[2][b] = ybn[3][b] = mk(0.0);
        }
        const bool ok = ev.grav == 1 ? sph_solver_nc_adj<1>(c, u, ev.rr, ev.rs, ev.ir, ev.is, ybn, yng, L, CL, G)
                                     : sph_solver_nc_adj<0>(c, u, ev.rr, ev.rs, ev.ir, ev.is, ybn, yng, L, CL, G);
        if (!ok) return false;
        for (int b = 0; b < 4; b++) {
            ysph[0][b] = yng[0][b];
            ysph[1][b] = yng[1][b];
            ysph[2][b] = mk(0.0);
        }
    }
    // grav(ir), the c0 coefficient of segment ir, through the correction
    if (ev.out == 2 && ev.cor != 0) {
        double gb = 0.0;
        for (int b = 0; b < 4; b++)
            gb += re(ybo[0][b] * (-2.0 * ysph[0][b] / ev.rr)) + re(ybo[1][b] * (zeta * ysph[0][b] / ev.rr));
        double vb[NPARAM];
        for (int p = 0; p < NPARAM; p++) vb[p] = 0.0;
        vb[P_GRAV] = gb;
        G.add(ev.ir, 0.0, vb);
    }
    if (ev.out == 1) {
        const cd f = imul(w);
        for (int b = 0; b < 4; b++)
            for (int a = 0; a < 3; a++) ysph[a][b] = f * ysph[a][b];
    } else if (ev.out == 2) {
        if (ev.cor == 0) {
            for (int b = 0; b < 4; b++)
                for (int a = 0; a < 3; a++) ysph[a][b] = mw2 * ysph[a][b];
        } else {
            for (int b = 0; b < 4; b++) {
                const cd c1 = (-((double)(l + 1) * ysph[2][b] + (2.0 * gr) * ysph[0][b])) / ev.rr;
                const cd c2 = (zeta * (ysph[2][b] + gr * ysph[0][b])) / ev.rr;
                ysph[0][b] = mw2 * ysph[0][b] + c1;
                ysph[1][b] = mw2 * ysph[1][b] + c2;
            }
        }
    }
    cd svsb[5][6];
    for (int q = 0; q < 5; q++)
        for (int b = 0; b < 6; b++) svsb[q][b] = mk(0.0);
    for (int q = 0; q < 5; q++) {
        const cd gu = uub[q] / ev.rr, gv = vvb[q] / zr;
        for (int b = 0; b < 4; b++) svsb[q][col[b]] = svsb[q][col[b]] + gu * ysph[0][b] + gv * ysph[1][b];
    }
    source_adj(c, u, ev.is, ev.rs, ev.mm, nullptr, svsb, G);
    return true;
}

}  // namespace YSG_VARIANT
}  // namespace ysg
