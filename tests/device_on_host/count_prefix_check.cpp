// count_prefix_check.cpp -- the count-only solve of the pair scheduler
// (ysg_solvers.cuh compiled with YSG_COUNT_ONLY), with the per-frequency
// prefix table of whole-interval step counts (k_step_prefix in
// k_schedule.cu, restated here on the host) against the interval-by-
// interval loop: every pair of the event, every system class's count must
// be equal.
//
//     count_prefix_check <yspec parameter file>
//
// It also compares every start-level search the drivers make with the
// search in its direct form (the quotients formed at every visit).
// Prints the pairs compared and the mismatches; exit status 0 if none.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "yspec_gpu.h"
#include "yspec_host.h"
#include "ysg_solvers.cuh"

using namespace ysg;

namespace {

// The start-level search of module_start.f90:14-178 as the solver formed it
// before the knot records carried 1/v^2 and r^2: both quotients per
// evaluation, every knot's q evaluated twice in the decay sum.
int start_level_direct(const Knot* kn, int l, double w, int i1, int i2, int wt)
{
    int isign = (i2 >= i1) ? 1 : -1;
    double pp = (double)(float)(l * (l + 1)) / (w * w);
    int j = i2;
    for (int i = i1; isign == 1 ? i <= i2 : i >= i2; i += isign) {
        double v = wt == 1 ? kn[i].beta : kn[i].alpha;
        double q1 = 1.0 / (v * v) - pp / (kn[i].r * kn[i].r);
        if (isign == 1) {
            if (q1 > 0.0) { j = std::max(i1, i - 1); break; }
        } else {
            if (q1 < 0.0) { j = i; break; }
        }
    }
    int is = j;
    int lo = std::min(i1, i2);
    if (is == lo) return is;
    int j1 = is;
    is = lo;
    double sum = 0.0;
    for (int i = j1; i >= lo + 1; i--) {
        double v1 = wt == 1 ? kn[i].beta : kn[i].alpha;
        double v2 = wt == 1 ? kn[i - 1].beta : kn[i - 1].alpha;
        double q1 = 1.0 / (v1 * v1) - pp / (kn[i].r * kn[i].r);
        double q2 = 1.0 / (v2 * v2) - pp / (kn[i - 1].r * kn[i - 1].r);
        if (q1 > 0.0 || q2 > 0.0) {
            sum = 0.0;
        } else {
            q1 = std::sqrt(-q1);
            q2 = std::sqrt(-q2);
            sum = sum + ((0.5 * w) * (q1 + q2)) * (kn[i].r - kn[i - 1].r);
        }
        if (sum > TOL_START) { is = i - 1; break; }
    }
    return is;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    ysh_params P;
    if (ysh_read_params(argv[1], &P)) return 2;
    ysh_model* m = nullptr;
    if (ysh_read_model(P.model_file, &m)) return 2;
    ysg_model v;
    ysh_model_view(m, &v);
    ysh_event E;
    if (ysh_event_setup(m, &P, &E)) return 2;
    const int n = v.nknot;
    std::vector<Knot> kn((size_t)n + 2);
    std::memset(kn.data(), 0, kn.size() * sizeof(Knot));
    for (int i = 0; i < n; i++) {
        kn[(size_t)i + 1].r = v.r[i];
        kn[(size_t)i + 1].alpha = v.alpha[i];
        kn[(size_t)i + 1].beta = v.beta[i];
        for (int p = 0; p < NPARAM; p++) {
            kn[(size_t)i + 1].v[p][0] = v.val[p][i];
            kn[(size_t)i + 1].v[p][1] = v.cs[p][i];
        }
        knot_derive(kn[(size_t)i + 1]);
    }
    std::vector<Seg> sg((size_t)n + 1);
    std::memset(sg.data(), 0, sg.size() * sizeof(Seg));
    ModelHdr mh;
    std::memset(&mh, 0, sizeof mh);
    mh.nknot = n;
    mh.nic = v.nic;
    mh.noc = v.noc;
    mh.nsl = v.nsl;
    mh.ocean = v.ocean;
    mh.fic = v.fic;
    int ia = 1;
    for (int i = 2; i <= n; i++)
        if (v.alpha[i - 1] < v.alpha[ia - 1]) ia = i;
    int ib = v.noc + 1;
    for (int i = v.noc + 2; i <= v.nsl; i++)
        if (v.beta[i - 1] < v.beta[ib - 1]) ib = i;
    mh.imin_alpha = ia;
    mh.imin_beta = ib;
    mh.tref = v.tref;
    mh.pibigg = v.pibigg;
    mh.fre_norm = v.fre_norm;
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
    ev.grav_ir = v.val[P_GRAV][e.ir - 1];
    for (int i = 0; i < 6; i++) ev.mm[i] = e.mm[i];
    long long pairs = 0, bad = 0, levels = 0, bad_levels = 0;
    std::vector<int> row((size_t)n + 1);
    for (int j = 1; j <= ev.nw; j++) {
        // the prefix row of k_step_prefix
        Ctx c;
        std::memset(&c, 0, sizeof c);
        c.kn = kn.data();
        c.mh = &mh;
        set_omega(c, omega_of(ev, j));
        int sum = 0;
        row[0] = row[1] = 0;
        for (int i = 1; i <= n - 1; i++) {
            const double h = kn[(size_t)i + 1].r - kn[(size_t)i].r;
            if (h != 0.0) sum += 1 + (int)fmin(floor(fabs(h) / steps(c, i)), 4194304.0);
            row[(size_t)i + 1] = sum;
        }
        // every start-level search the drivers make, against the direct form
        for (int l = ev.lmin; l <= ev.lmax; l++) {
            const double wr = c.omega.x;
            const int args[4][3] = {{mh.noc + 1, ev.is, 1}, {mh.nic + 1, mh.noc, 2}, {2, mh.nic, 1}, {2, mh.nic, 2}};
            for (const auto& a : args) {
                levels++;
                if (start_level(c, l, wr, a[0], a[1], a[2]) != start_level_direct(kn.data(), l, wr, a[0], a[1], a[2]))
                    bad_levels++;
            }
        }
        for (int l = ev.lmin; l <= ev.lmax; l++)
            for (int part = 0; part < 2; part++) {
                if (part == 1 && l < 2) continue;
                unsigned cnt[2][NSYS];
                for (int way = 0; way < 2; way++) {
                    Ctx d;
                    std::memset(&d, 0, sizeof d);
                    d.kn = kn.data();
                    d.mh = &mh;
                    d.sg = sg.data();
                    d.pib = mh.pibigg;
                    d.ats = ev.ats;
                    d.pfx = way ? row.data() : nullptr;
                    cd out[NCOEF];
                    if (part == 1) pair_toroidal(d, ev, l, j, out + 10);
                    else if (l == 0) pair_radial(d, ev, j, out);
                    else pair_spheroidal(d, ev, l, j, out, out + 5);
                    for (int q = 0; q < NSYS; q++) cnt[way][q] = d.nst[q];
                }
                pairs++;
                if (std::memcmp(cnt[0], cnt[1], sizeof cnt[0]) != 0) {
                    if (bad < 10)
                        std::printf("mismatch l %d j %d part %d: class 6 %u vs %u, class 7 %u vs %u\n", l, j, part,
                                    cnt[0][6], cnt[1][6], cnt[0][7], cnt[1][7]);
                    bad++;
                }
            }
    }
    std::printf("start levels %lld differing %lld\n", levels, bad_levels);
    std::printf("pairs %lld mismatches %lld\n", pairs, bad);
    return bad == 0 && bad_levels == 0 ? 0 : 1;
}
