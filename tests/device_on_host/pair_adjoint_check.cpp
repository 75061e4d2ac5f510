// pair_adjoint_check.cpp -- the reverse sweep of single (omega, l) pairs
// (ysg_pair_adjoint.cuh) against the tangent-linear form of the same pair
// solve (the solver headers compiled with dual numbers), on the CPU.
//
//     pair_adjoint_check <yspec parameter file>
//
// For the event of the parameter file (host library: ysh_read_params,
// ysh_read_model, ysh_event_setup) and a set of pairs (l, j) covering the
// radial, toroidal and spheroidal solves, with a random weight vector w and
// a random model direction (knot values and spline second derivatives, the
// segments derived from them as the upload does), it compares
//     tangent: d/de Re(sum_q w_q coef_q(model + e direction)) at e = 0
//     adjoint: <dL/d(knot arrays), direction>, dL/d(segments) from the
//              reverse sweep mapped to the knot arrays.
// Prints one line per pair and the worst relative difference; exit status
// 0 if it is below 1e-9.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "yspec_gpu.h"
#include "yspec_host.h"
#include "ysg_pair_adjoint.cuh"

using namespace ysg;

namespace {

struct Tables {
    std::vector<Knot> kn;
    std::vector<Seg> sg;
    ModelHdr mh;
};

// the knot records, power-form segments and header the upload builds
void build(const ysg_model* m, Tables& T)
{
    const int n = m->nknot;
    T.kn.assign((size_t)n + 2, Knot{});
    std::memset(T.kn.data(), 0, T.kn.size() * sizeof(Knot));
    for (int i = 0; i < n; i++) {
        Knot& k = T.kn[(size_t)i + 1];
        k.r = m->r[i];
        k.alpha = m->alpha[i];
        k.beta = m->beta[i];
        for (int p = 0; p < NPARAM; p++) {
            k.v[p][0] = m->val[p][i];
            k.v[p][1] = m->cs[p][i];
        }
        knot_derive(k);
    }
    T.sg.assign((size_t)n + 1, Seg{});
    std::memset(T.sg.data(), 0, T.sg.size() * sizeof(Seg));
    for (int i = 1; i < n; i++) {
        Seg& s = T.sg[(size_t)i];
        const Knot &a = T.kn[(size_t)i], &b = T.kn[(size_t)i + 1];
        const double hh = b.r - a.r;
        s.r0 = a.r;
        for (int p = 0; p < NPARAM; p++) {
            s.c[p][0] = a.v[p][0];
            if (hh == 0.0) continue;
            s.c[p][1] = (b.v[p][0] - a.v[p][0]) / hh - hh * (2.0 * a.v[p][1] + b.v[p][1]) / 6.0;
            s.c[p][2] = 0.5 * a.v[p][1];
            s.c[p][3] = (b.v[p][1] - a.v[p][1]) / (6.0 * hh);
        }
    }
    T.sg[(size_t)n].r0 = T.kn[(size_t)n].r;
    for (int p = 0; p < NPARAM; p++) T.sg[(size_t)n].c[p][0] = T.kn[(size_t)n].v[p][0];
    ModelHdr& hd = T.mh;
    std::memset(&hd, 0, sizeof hd);
    hd.nknot = n;
    hd.nic = m->nic;
    hd.noc = m->noc;
    hd.nsl = m->nsl;
    hd.ocean = m->ocean;
    hd.fic = m->fic;
    int ia = 1;
    for (int i = 2; i <= n; i++)
        if (m->alpha[i - 1] < m->alpha[ia - 1]) ia = i;
    int ib = m->noc + 1;
    for (int i = m->noc + 2; i <= m->nsl; i++)
        if (m->beta[i - 1] < m->beta[ib - 1]) ib = i;
    hd.imin_alpha = ia;
    hd.imin_beta = ib;
    hd.tref = m->tref;
    hd.pibigg = m->pibigg;
    hd.fre_norm = m->fre_norm;
}

// d/de Re(sum_q w_q coef_q) along (dkn, dsg): the tangent-linear pair solve
double tangent_pair(const Tables& T, const std::vector<Knot>& dkn, const std::vector<Seg>& dsg,
                    const EventDev& ev, int l, int j, const cd* w)
{
    v_tangent::Ctx c;
    std::memset(&c, 0, sizeof c);
    c.kn = T.kn.data();
    c.mh = &T.mh;
    c.sg = T.sg.data();
    c.dkn = dkn.data();
    c.dsg = dsg.data();
    c.pib = T.mh.pibigg;
    c.ats = ev.ats;
    v_tangent::mcplx out[NCOEF];
    for (int q = 0; q < NCOEF; q++) out[q] = v_tangent::mcplx(mk(0.0));
    if (l == 0) {
        pair_radial(c, ev, j, out);
    } else {
        if (l > 1) pair_toroidal(c, ev, l, j, out + 10);
        pair_spheroidal(c, ev, l, j, out, out + 5);
    }
    double d = 0.0;
    for (int q = 0; q < NCOEF; q++) d += (w[q] * out[q].d).x;
    return d;
}

// dL/dc[i][p][k] -> dL/d(knot value), dL/d(spline second derivative),
// through the segment formulas of build()
void seg_to_knot(const Tables& T, const std::vector<double>& g, std::vector<double>& yb, std::vector<double>& ysb)
{
    const int n = T.mh.nknot;
    yb.assign((size_t)(n + 2) * NPARAM, 0.0);
    ysb.assign((size_t)(n + 2) * NPARAM, 0.0);
    for (int i = 1; i <= n; i++)
        for (int p = 0; p < NPARAM; p++) {
            const double* c = &g[((size_t)i * NPARAM + p) * 4];
            yb[(size_t)i * NPARAM + p] += c[0];
            if (i == n) continue;
            const double h = T.kn[i + 1].r - T.kn[i].r;
            if (h == 0.0) continue;
            yb[(size_t)(i + 1) * NPARAM + p] += c[1] / h;
            yb[(size_t)i * NPARAM + p] -= c[1] / h;
            ysb[(size_t)i * NPARAM + p] += -c[1] * h / 3.0 + 0.5 * c[2] - c[3] / (6.0 * h);
            ysb[(size_t)(i + 1) * NPARAM + p] += -c[1] * h / 6.0 + c[3] / (6.0 * h);
        }
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <parameter file>\n", argv[0]);
        return 2;
    }
    ysh_params P;
    if (ysh_read_params(argv[1], &P)) return 2;
    ysh_model* m = nullptr;
    if (ysh_read_model(P.model_file, &m)) return 2;
    ysg_model view;
    ysh_model_view(m, &view);
    Tables T;
    build(&view, T);
    ysh_event E;
    if (ysh_event_setup(m, &P, &E)) return 2;
    const ysg_event& e = E.ev;
    EventDev ev{};
    ev.lmin = e.lmin;
    ev.lmax = e.lmax;
    ev.nw = e.nw;
    ev.is = e.is;
    ev.ir = e.ir;
    ev.ats = e.ats;
    ev.grav = e.grav;
    ev.out = e.out;
    ev.cor = e.cor;
    ev.nr = e.nr;
    ev.jofs = 0;
    ev.jstride = 1;
    ev.rs = e.rs;
    ev.rr = e.rr;
    ev.ep = e.ep;
    ev.wmin = e.wmin;
    ev.dw = e.dw;
    ev.grav_ir = view.val[P_GRAV][e.ir - 1];
    for (int i = 0; i < 6; i++) ev.mm[i] = e.mm[i];
    const int n = T.mh.nknot;
    std::mt19937_64 rng(9);
    std::normal_distribution<double> nd;
    // a random direction in the knot arrays and the segments derived from it
    std::vector<Knot> dkn(T.kn.size());
    std::memset(dkn.data(), 0, dkn.size() * sizeof(Knot));
    for (int i = 1; i <= n; i++)
        for (int p = 0; p < NPARAM; p++) {
            dkn[i].v[p][0] = nd(rng) * std::fabs(T.kn[i].v[p][0]) * 1e-2;
            dkn[i].v[p][1] = nd(rng) * 1e-2;
        }
    std::vector<Seg> dsg(T.sg.size());
    std::memset(dsg.data(), 0, dsg.size() * sizeof(Seg));
    for (int i = 1; i < n; i++) {
        const double hh = T.kn[i + 1].r - T.kn[i].r;
        for (int p = 0; p < NPARAM; p++) {
            dsg[i].c[p][0] = dkn[i].v[p][0];
            if (hh == 0.0) continue;
            dsg[i].c[p][1] = (dkn[i + 1].v[p][0] - dkn[i].v[p][0]) / hh -
                             hh * (2.0 * dkn[i].v[p][1] + dkn[i + 1].v[p][1]) / 6.0;
            dsg[i].c[p][2] = 0.5 * dkn[i].v[p][1];
            dsg[i].c[p][3] = (dkn[i + 1].v[p][1] - dkn[i].v[p][1]) / (6.0 * hh);
        }
    }
    for (int p = 0; p < NPARAM; p++) dsg[n].c[p][0] = dkn[n].v[p][0];
    // unit directions of the start and source vectors
    std::vector<std::vector<Knot>> ukn(NPARAM, std::vector<Knot>(T.kn.size()));
    std::vector<std::vector<Seg>> usg(NPARAM, std::vector<Seg>(T.sg.size()));
    UnitDirs U;
    for (int p = 0; p < NPARAM; p++) {
        std::memset(ukn[p].data(), 0, ukn[p].size() * sizeof(Knot));
        std::memset(usg[p].data(), 0, usg[p].size() * sizeof(Seg));
        for (size_t i = 0; i < ukn[p].size(); i++) ukn[p][i].v[p][0] = 1.0;
        for (size_t i = 0; i < usg[p].size(); i++) usg[p][i].c[p][0] = 1.0;
        U.kn[p] = ukn[p].data();
        U.sg[p] = usg[p].data();
    }
    const int N = 14, nmax = 100000, gmax = 200000;
    std::vector<cd> ly((size_t)nmax * N), gy((size_t)gmax * 4);
    std::vector<double> lx(nmax), lh(nmax), lf(nmax), gr(gmax);
    std::vector<int> lil(nmax), gi(gmax);
    StepLog L{ly.data(), lx.data(), lh.data(), lil.data(), lf.data(), nmax, 1};
    std::vector<cd> cy((size_t)nmax * N);
    std::vector<double> cx(nmax), ch(nmax), cf(nmax);
    std::vector<int> cil(nmax);
    StepLog CL{cy.data(), cx.data(), ch.data(), cil.data(), cf.data(), nmax, 1};
    GridLog GL{gy.data(), gr.data(), gi.data(), gmax, 1};
    const int pairs[][2] = {{0, 3},      {0, ev.nw / 2}, {0, ev.nw},     {1, ev.nw},      {2, ev.nw},
                            {1, 3},      {2, 10},        {5, 40},        {20, ev.nw / 2}, {60, ev.nw},
                            {150, ev.nw}, {ev.lmax, ev.nw / 3}};
    double worst = 0.0;
    int bad = 0;
    for (const auto& pr : pairs) {
        const int l = pr[0], j = pr[1];
        if (l > ev.lmax || j < 1 || j > ev.nw) continue;
        cd w[NCOEF];
        for (int q = 0; q < NCOEF; q++) w[q] = mk(nd(rng), nd(rng));
        const double dt = tangent_pair(T, dkn, dsg, ev, l, j, w);
        std::vector<double> g((size_t)(n + 1) * NPARAM * 4, 0.0);
        SegGrad G;
        G.init(g.data());
        primal::Ctx c;
        std::memset(&c, 0, sizeof c);
        c.kn = T.kn.data();
        c.mh = &T.mh;
        c.sg = T.sg.data();
        c.pib = T.mh.pibigg;
        c.ats = ev.ats;
        bool ok = true;
        if (l == 0) {
            ok = pair_radial_adj(c, U, ev, j, w, L, CL, GL, G);
        } else {
            if (l > 1) ok = pair_toroidal_adj(c, U, ev, l, j, w + 10, L, CL, G);
            ok = ok && pair_spheroidal_adj(c, U, ev, l, j, w, w + 5, L, CL, G);
        }
        G.flush();
        std::vector<double> yb, ysb;
        seg_to_knot(T, g, yb, ysb);
        double da = 0.0;
        for (int i = 1; i <= n; i++)
            for (int p = 0; p < NPARAM; p++)
                da += yb[(size_t)i * NPARAM + p] * dkn[i].v[p][0] + ysb[(size_t)i * NPARAM + p] * dkn[i].v[p][1];
        const double rel = std::fabs(da - dt) / std::fabs(dt);
        if (!ok) bad++;
        worst = std::max(worst, ok ? rel : 1.0);
        std::printf("l %4d j %4d ok %d adjoint % .15e tangent % .15e rel %.2e\n", l, j, ok ? 1 : 0, da, dt, rel);
    }
    std::printf("worst %.3e\n", worst);
    return (bad == 0 && worst < 1e-9) ? 0 : 1;
}
