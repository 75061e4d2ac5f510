// bvec_transpose_check.cpp -- the spheroidal pair solve of the batched form
// (shared-memory stages: only the response rows a pair uses, each from one
// backward integration of the transposed b-vector system) against the
// plain form (four forward b-vector integrations, one per source jump), on
// the CPU.
//
//     bvec_transpose_check <yspec parameter file> [frequency stride]
//
// For the event of the parameter file (host library: ysh_read_params,
// ysh_read_model, ysh_event_setup) and every degree l >= 1 at every
// stride-th frequency, it compares the ten spheroidal coefficients
// uu(1:5), vv(1:5) of the two forms: the error of a pair is the largest
// difference over the largest magnitude of the plain form's ten.  It also
// checks one transposed Cash-Karp step against the forward step's matrix.
// Prints the worst pair error; exit status 0 if it is below 1e-10.
//
// The two forms share their complex type, so they cannot sit in one
// translation unit: the file is compiled three times, with BVT_PART=1 (the
// shared-memory form), BVT_PART=2 (the plain form) and without (main), and
// the objects are linked together.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "yspec_gpu.h"
#include "yspec_host.h"

#ifndef BVT_PART
#define BVT_PART 0
#endif
#if BVT_PART == 1
#define YSG_SMEM_STAGES 1
#endif
#if BVT_PART != 0
#include "ysg_solvers.cuh"
#else
#include "ysg_model.cuh"
#endif

using namespace ysg;

struct Tables {
    std::vector<Knot> kn;
    std::vector<Seg> sg;
    ModelHdr mh;
};

// the spheroidal coefficients uu(1:5), vv(1:5) of pair (l, j) in one form
void pair_sph_smem(const Tables& T, const EventDev& ev, int l, int j, cd* out, cd* slab);
void pair_sph_plain(const Tables& T, const EventDev& ev, int l, int j, cd* out);
double step_check(const Tables& T, const EventDev& ev, cd* slab);

#if BVT_PART != 0
namespace {
template <class C>
void init_ctx(C& c, const Tables& T, const EventDev& ev)
{
    std::memset(&c, 0, sizeof c);
    c.kn = T.kn.data();
    c.mh = &T.mh;
    c.sg = T.sg.data();
    c.pib = T.mh.pibigg;
    c.ats = ev.ats;
}
double cabs_(cd a) { return std::hypot(a.x, a.y); }
}  // namespace
#endif

#if BVT_PART == 1
void pair_sph_smem(const Tables& T, const EventDev& ev, int l, int j, cd* out, cd* slab)
{
    Ctx c;
    init_ctx(c, T, ev);
    c.kb = slab;
    pair_spheroidal(c, ev, l, j, out, out + 5);
}

// One transposed step against the forward step's matrix, at a mantle radius:
// w . (M e_j) for every unit vector e_j against (M^T w)_j.
double step_check(const Tables& T, const EventDev& ev, cd* slab)
{
    Ctx c;
    init_ctx(c, T, ev);
    c.kb = slab;
    set_l(c, 40);
    set_omega(c, omega_of(ev, ev.nw / 2 > 0 ? ev.nw / 2 : 1));
    const int il = T.mh.nsl - 3;
    c.il = il;
    const double x = T.kn[il].r, h = 0.3 * (T.kn[il + 1].r - T.kn[il].r);
    std::mt19937_64 rng(3);
    std::normal_distribution<double> nd;
    cd w[14], wt[14];
    for (int k = 0; k < 14; k++) w[k] = wt[k] = cd{nd(rng), nd(rng)};
    rkck_step_loop_T<BvecSolidGTr>(c, wt, x, h);
    double worst = 0.0, scale = 0.0;
    for (int j = 0; j < 14; j++) {
        cd y[14];
        for (int k = 0; k < 14; k++) y[k] = mk(k == j ? 1.0 : 0.0);
        rkck_step_loop<BvecSolidG>(c, y, x, h);
        cd dot = mk(0.0);
        for (int k = 0; k < 14; k++) dot = dot + w[k] * y[k];
        worst = std::fmax(worst, cabs_(dot - wt[j]));
        scale = std::fmax(scale, cabs_(wt[j]));
    }
    return worst / scale;
}
#elif BVT_PART == 2
void pair_sph_plain(const Tables& T, const EventDev& ev, int l, int j, cd* out)
{
    Ctx c;
    init_ctx(c, T, ev);
    pair_spheroidal(c, ev, l, j, out, out + 5);
}
#else

namespace {

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

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <parameter file> [frequency stride]\n", argv[0]);
        return 2;
    }
    const int stride = argc > 2 ? std::atoi(argv[2]) : 1;
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

    // lane 0 of a warp's interleaved slab: entry e at slab[e * KS]
    std::vector<cd> slab((size_t)4 * 14 * 32);
    const double step_err = step_check(T, ev, slab.data());
    std::printf("transposed step %.3e\n", step_err);

    double worst = 0.0;
    long long pairs = 0;
    for (int j = 1; j <= ev.nw; j += stride)
        for (int l = ev.lmin > 1 ? ev.lmin : 1; l <= ev.lmax; l++) {
            cd ua[10], ub[10];
            pair_sph_smem(T, ev, l, j, ua, slab.data());
            pair_sph_plain(T, ev, l, j, ub);
            double d = 0.0, s = 0.0;
            for (int q = 0; q < 10; q++) {
                d = std::fmax(d, std::hypot(ua[q].x - ub[q].x, ua[q].y - ub[q].y));
                s = std::fmax(s, std::hypot(ub[q].x, ub[q].y));
            }
            const double err = s > 0.0 ? d / s : d;
            if (!(err <= worst)) worst = err;
            pairs++;
        }
    std::printf("pairs %lld worst %.3e\n", pairs, worst);
    return (step_err < 1e-12 && worst < 1e-10) ? 0 : 1;
}
#endif
