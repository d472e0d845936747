// gromos_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// FP64 CPU restatement of the gromos-rs nonbonded hot path.  Every function
// names the reference file:line it follows (paths relative to the gromos-rs
// repository).  Compile with -ffp-contract=off: the reference is Rust, which
// never fuses a*b+c, and the operation order below is the reference's.
//
// Additions that the reference does not have are marked "ADDITION": the
// per-energy-group attribution of every energy term (the reference stores
// group matrices but never fills them, configuration.rs:151-154), and an
// std::thread fold/reduce mode used only to time the CPU baseline.
#include "gromos_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <set>
#include <atomic>
#include <thread>
#include <vector>

namespace {

struct V3 {
    double x, y, z;
};
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double comp(const V3& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
// glam DVec3::length_squared = dot(self, self) = (x*x + y*y) + z*z
inline double len2(V3 r) { return r.x * r.x + r.y * r.y + r.z * r.z; }
// f64::powi: exponentiation by squaring (the expansion Rust/LLVM use).
inline double powi(double a, int b) {
    bool recip = b < 0;
    unsigned e = recip ? unsigned(-b) : unsigned(b);
    double r = 1.0;
    while (true) {
        if (e & 1u) r *= a;
        e >>= 1;
        if (e == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

// Rectangular / Vacuum periodicity (crates/gromos-core/src/math.rs:20-74).
struct Boundary {
    int type = 1;  // 0 vacuum, 1 rectangular
    V3 box{0, 0, 0}, half{0, 0, 0}, inv{0, 0, 0};
    void set(int t, const double b[3]) {
        type = t;
        box = {b[0], b[1], b[2]};
        half = box * 0.5;                                         // math.rs:52
        inv = {1.0 / box.x, 1.0 / box.y, 1.0 / box.z};            // math.rs:53 recip()
    }
    // math.rs:60-68: r = (ri - rj) - box * round((ri - rj) * inv_box)
    V3 nearest_image(V3 ri, V3 rj) const {
        V3 r = ri - rj;
        if (type == 0) return r;
        V3 k{std::round(r.x * inv.x), std::round(r.y * inv.y), std::round(r.z * inv.z)};
        return {r.x - box.x * k.x, r.y - box.y * k.y, r.z - box.z * k.z};
    }
};

struct CRF {
    double crf_cut, crf_2cut3i, crf_cut3i, cutoff_sq;
};

// CRFParameters::new (crates/gromos-forces/src/nonbonded/params.rs:78-96).
CRF make_crf(double cutoff, double epsilon, double rf_epsilon, double rf_kappa) {
    double kappa_cut = rf_kappa * cutoff;
    double kappa_cut2 = kappa_cut * kappa_cut;
    double crf = (2.0 * (epsilon - rf_epsilon) * (1.0 + kappa_cut) - rf_epsilon * kappa_cut2) /
                 ((epsilon + 2.0 * rf_epsilon) * (1.0 + kappa_cut) + rf_epsilon * kappa_cut2);
    double cut3i = 1.0 / (cutoff * cutoff * cutoff);
    CRF c;
    c.crf_cut3i = crf * cut3i;
    c.crf_2cut3i = c.crf_cut3i / 2.0;
    c.crf_cut = (1.0 - crf / 2.0) / cutoff;
    c.cutoff_sq = cutoff * cutoff;
    return c;
}

struct LJ {
    double c6, c12, cs6, cs12;
};

// Lambda-dependent parameters (perturbed.rs:12-101).
struct LambdaParams {
    double a_lj_n, b_lj_n, a_crf_n, b_crf_n;
    double a_lj_n1, b_lj_n1, a_crf_n1, b_crf_n1;
    double a_ljs, b_ljs, a_ljs2, b_ljs2;
    double a_crfs, b_crfs, a_crfs2, b_crfs2;
    int n;
};

LambdaParams from_lambda(double lj, double ljs, double crf, double crfs, double dlj, double dljs,
                         double dcrf, double dcrfs, int n) {
    LambdaParams p;
    p.a_lj_n = powi(1.0 - lj, n);  // (1-λ)^n
    p.a_crf_n = powi(1.0 - crf, n);
    p.b_lj_n = powi(lj, n);
    p.b_crf_n = powi(crf, n);
    p.a_lj_n1 = powi(1.0 - lj, n - 1) * dlj;
    p.a_crf_n1 = powi(1.0 - crf, n - 1) * dcrf;
    p.b_lj_n1 = powi(lj, n - 1) * dlj;
    p.b_crf_n1 = powi(crf, n - 1) * dcrf;
    p.a_ljs = (1.0 - ljs) * dljs;
    p.a_crfs = (1.0 - crfs) * dcrfs;
    p.b_ljs = ljs * dljs;
    p.b_crfs = crfs * dcrfs;
    p.a_ljs2 = (1.0 - ljs) * (1.0 - ljs);
    p.a_crfs2 = (1.0 - crfs) * (1.0 - crfs);
    p.b_ljs2 = ljs * ljs;
    p.b_crfs2 = crfs * crfs;
    p.n = n;
    return p;
}

// Per-thread accumulator (ForceStorage, params.rs:100-138) plus the
// energy-group matrices (ADDITION).
struct Storage {
    std::vector<V3> f;
    double e_lj = 0, e_crf = 0;
    double vir[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    int G = 1;
    std::vector<double> g_lj, g_crf;  // G*G, [min][max]
    void init(int n, int g) {
        f.assign(n, V3{0, 0, 0});
        G = g;
        g_lj.assign(size_t(g) * g, 0.0);
        g_crf.assign(size_t(g) * g, 0.0);
        clear_scalars();
    }
    void clear_scalars() {
        e_lj = e_crf = 0;
        std::memset(vir, 0, sizeof(vir));
    }
    void clear() {
        std::fill(f.begin(), f.end(), V3{0, 0, 0});
        std::fill(g_lj.begin(), g_lj.end(), 0.0);
        std::fill(g_crf.begin(), g_crf.end(), 0.0);
        clear_scalars();
    }
    // ForceStorage::merge (params.rs:126-137)
    void merge(const Storage& o) {
        for (size_t i = 0; i < f.size(); ++i) f[i] = f[i] + o.f[i];
        e_lj += o.e_lj;
        e_crf += o.e_crf;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) vir[a][b] += o.vir[a][b];
        for (size_t k = 0; k < g_lj.size(); ++k) {
            g_lj[k] += o.g_lj[k];
            g_crf[k] += o.g_crf[k];
        }
    }
    inline void group_add(int gi, int gj, double elj, double ecrf) {
        int a = gi < gj ? gi : gj, b = gi < gj ? gj : gi;
        g_lj[size_t(a) * G + b] += elj;
        g_crf[size_t(a) * G + b] += ecrf;
    }
};

// lj_crf_interaction (crates/gromos-forces/src/nonbonded/innerloops.rs:21-55).
inline void lj_crf_interaction(V3 r, double c6, double c12, double q_prod, const CRF& crf,
                               double& f_mag, double& e_lj, double& e_crf) {
    double r2 = len2(r);
    if (r2 < 1e-10) {
        f_mag = e_lj = e_crf = 0.0;
        return;
    }
    double inv_r2 = 1.0 / r2;
    double inv_r6 = inv_r2 * inv_r2 * inv_r2;
    e_lj = (c12 * inv_r6 - c6) * inv_r6;
    double f_lj = (12.0 * c12 * inv_r6 - 6.0 * c6) * inv_r6 * inv_r2;
    double inv_r = std::sqrt(inv_r2);
    e_crf = q_prod * (inv_r - crf.crf_2cut3i * r2 - crf.crf_cut);
    double f_crf = q_prod * (inv_r * inv_r2 + crf.crf_cut3i);
    f_mag = f_lj + f_crf;
}

using Pair = std::pair<int32_t, int32_t>;

// Dynamic-schedule parallel for over [0, n) on `nth` std::threads; body(k, tid).
template <class F>
void parallel_for(int nth, size_t n, F body) {
    if (nth <= 1) {
        for (size_t k = 0; k < n; ++k) body(k, 0);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nth; ++t)
        th.emplace_back([&, t] {
            for (size_t k = next.fetch_add(1); k < n; k = next.fetch_add(1)) body(k, t);
        });
    for (auto& x : th) x.join();
}

struct Topo {
    const orc_topology* t;
    int n;
    std::vector<std::vector<int>> cg_atoms;
    std::vector<int> egroup;
    int G = 1;
    bool has_o14 = false;
    std::vector<LJ> lj;
    int nt;

    explicit Topo(const orc_topology* tp) : t(tp) {
        n = tp->n_atoms;
        cg_atoms.resize(tp->n_cg);
        for (int c = 0; c < tp->n_cg; ++c)
            for (int a = tp->cg_offsets[c]; a < tp->cg_offsets[c + 1]; ++a) cg_atoms[c].push_back(a);
        egroup.assign(n, 0);
        G = tp->n_egroups > 0 ? tp->n_egroups : 1;
        if (tp->egroup)
            for (int a = 0; a < n; ++a) egroup[a] = tp->egroup[a];
        has_o14 = tp->o14_off && tp->o14_off[n] > 0;
        nt = tp->n_types;
        lj.resize(size_t(nt) * nt);
        for (size_t k = 0; k < lj.size(); ++k)
            lj[k] = {tp->lj[4 * k], tp->lj[4 * k + 1], tp->lj[4 * k + 2], tp->lj[4 * k + 3]};
    }
    const LJ& ljp(int ti, int tj) const { return lj[size_t(ti) * nt + tj]; }  // params.rs:50-52
    bool excl_contains(int i, int j) const {
        const int32_t* b = t->excl + t->excl_off[i];
        const int32_t* e = t->excl + t->excl_off[i + 1];
        return std::binary_search(b, e, j);
    }
    bool o14_contains(int i, int j) const {
        for (int k = t->o14_off[i]; k < t->o14_off[i + 1]; ++k)
            if (t->o14[k] == j) return true;
        return false;
    }
    // Topology::is_excluded_or_14 (topology.rs:853-864)
    bool is_excluded_or_14(int i, int j) const {
        if (excl_contains(i, j) || excl_contains(j, i)) return true;
        if (has_o14 && (o14_contains(i, j) || o14_contains(j, i))) return true;
        return false;
    }
    // ChargeGroup::center_of_geometry (topology.rs:408-417): sum from ZERO, / len
    V3 cog(int c, const V3* pos) const {
        const auto& at = cg_atoms[c];
        if (at.empty()) return {0, 0, 0};
        V3 s{0, 0, 0};
        for (int a : at) s = s + pos[a];
        double len = double(at.size());
        return {s.x / len, s.y / len, s.z / len};
    }
    bool perturbed(int a) const { return t->pert_idx && t->pert_idx[a] >= 0; }
};

struct Lists {
    std::vector<Pair> l[4];  // solute_short, solute_long, solvent_short, solvent_long
    void clear() {
        for (auto& v : l) v.clear();
    }
};

// StandardPairlistAlgorithm::update_chargegroup_based (pairlist.rs:183-442).
void pairlist_standard(const Topo& T, const Boundary& bc, const V3* pos, double rcs, double rcl,
                       double skin, Lists& L) {
    const orc_topology* t = T.t;
    int ncg = t->n_cg, nsol = t->n_solute_cg;
    double c2s = (rcs + skin) * (rcs + skin);  // pairlist.rs:192 powi(2)
    double c2l = (rcl + skin) * (rcl + skin);
    std::vector<V3> cog(nsol);
    for (int c = 0; c < nsol; ++c) cog[c] = T.cog(c, pos);
    auto& ss = L.l[0];
    auto& sl = L.l[1];
    auto& vs = L.l[2];
    auto& vl = L.l[3];
    for (int cg1 = 0; cg1 < nsol; ++cg1) {
        const auto& a1s = T.cg_atoms[cg1];
        for (size_t ai = 0; ai < a1s.size(); ++ai)  // intra-CG (pairlist.rs:239-249)
            for (size_t aj = ai + 1; aj < a1s.size(); ++aj)
                if (!T.is_excluded_or_14(a1s[ai], a1s[aj])) ss.push_back({a1s[ai], a1s[aj]});
        for (int cg2 = cg1 + 1; cg2 < nsol; ++cg2) {  // solute-solute (:252-301)
            double d2 = len2(bc.nearest_image(cog[cg1], cog[cg2]));
            if (d2 > c2l) continue;
            if (d2 > c2s) {
                for (int a1 : a1s)
                    for (int a2 : T.cg_atoms[cg2]) sl.push_back({a1, a2});
                continue;
            }
            for (int a1 : a1s)
                for (int a2 : T.cg_atoms[cg2])
                    if (!T.is_excluded_or_14(a1, a2)) ss.push_back({a1, a2});
        }
        for (int cg2 = nsol; cg2 < ncg; ++cg2) {  // solute-solvent (:304-350)
            int fa = T.cg_atoms[cg2][0];
            double d2 = len2(bc.nearest_image(cog[cg1], pos[fa]));
            if (d2 > c2l) continue;
            auto& dst = d2 > c2s ? sl : ss;
            for (int a1 : a1s)
                for (int a2 : T.cg_atoms[cg2]) dst.push_back({a1, a2});
        }
    }
    for (int cg1 = nsol; cg1 < ncg; ++cg1) {  // solvent-solvent (:359-415)
        int f1 = T.cg_atoms[cg1][0];
        for (int cg2 = cg1 + 1; cg2 < ncg; ++cg2) {
            int f2 = T.cg_atoms[cg2][0];
            double d2 = len2(bc.nearest_image(pos[f1], pos[f2]));
            if (d2 > c2l) continue;
            if (d2 > c2s) {
                for (int a1 : T.cg_atoms[cg1])
                    for (int a2 : T.cg_atoms[cg2]) vl.push_back({a1, a2});
                continue;
            }
            vs.push_back({f1, f2});
        }
    }
}

// process_cg_pair (pairlist.rs:698-777).
void process_cg_pair(int cga, int cgb, const Topo& T, const Boundary& bc, const V3* pos,
                     const std::vector<V3>& cog, double c2s, double c2l, Lists& L) {
    int nsol = T.t->n_solute_cg;
    int cg1 = std::min(cga, cgb), cg2 = std::max(cga, cgb);
    if (cg2 < nsol) {
        double d2 = len2(bc.nearest_image(cog[cg1], cog[cg2]));
        if (d2 > c2l) return;
        if (d2 > c2s) {
            for (int a1 : T.cg_atoms[cg1])
                for (int a2 : T.cg_atoms[cg2]) L.l[1].push_back({a1, a2});
        } else {
            for (int a1 : T.cg_atoms[cg1])
                for (int a2 : T.cg_atoms[cg2])
                    if (!T.is_excluded_or_14(a1, a2)) L.l[0].push_back({a1, a2});
        }
    } else if (cg1 < nsol) {
        int fa = T.cg_atoms[cg2][0];
        double d2 = len2(bc.nearest_image(cog[cg1], pos[fa]));
        if (d2 > c2l) return;
        auto& dst = d2 > c2s ? L.l[1] : L.l[0];
        for (int a1 : T.cg_atoms[cg1])
            for (int a2 : T.cg_atoms[cg2]) dst.push_back({a1, a2});
    } else {
        int f1 = T.cg_atoms[cg1][0], f2 = T.cg_atoms[cg2][0];
        double d2 = len2(bc.nearest_image(pos[f1], pos[f2]));
        if (d2 > c2l) return;
        if (d2 > c2s) {
            for (int a1 : T.cg_atoms[cg1])
                for (int a2 : T.cg_atoms[cg2]) L.l[3].push_back({a1, a2});
        } else {
            L.l[2].push_back({f1, f2});
        }
    }
}

// CellListPairlistAlgorithm::update_cell_list (pairlist.rs:537-655) with
// grid_dim_for_axis / cell_index / neighbor_cells (:658-692).  Neighbour
// cells are visited in sorted order (the reference's HashSet order is
// unspecified, so only the pair SET is defined).
void pairlist_cell(const Topo& T, const Boundary& bc, const V3* pos, double rcs, double rcl,
                   double skin, int nthreads, Lists& L) {
    const orc_topology* t = T.t;
    int ncg = t->n_cg, nsol = t->n_solute_cg;
    if (ncg == 0) return;
    double c2s = (rcs + skin) * (rcs + skin), c2l = (rcl + skin) * (rcl + skin);
    double minc = rcl + skin;
    std::vector<V3> cog(nsol);
    for (int c = 0; c < nsol; ++c) cog[c] = T.cog(c, pos);
    for (int c = 0; c < nsol; ++c) {
        const auto& at = T.cg_atoms[c];
        for (size_t ai = 0; ai < at.size(); ++ai)
            for (size_t aj = ai + 1; aj < at.size(); ++aj)
                if (!T.is_excluded_or_14(at[ai], at[aj])) L.l[0].push_back({at[ai], at[aj]});
    }
    std::vector<V3> ref(ncg);
    for (int c = 0; c < ncg; ++c) ref[c] = c < nsol ? cog[c] : pos[T.cg_atoms[c][0]];
    auto gdim = [&](double len) -> long {
        if (minc <= 0.0 || len <= 0.0) return 1;
        long g = long(std::floor(len / minc));
        return g < 1 ? 1 : g;
    };
    long gd[3] = {gdim(bc.box.x), gdim(bc.box.y), gdim(bc.box.z)};
    double cs[3] = {bc.box.x / double(gd[0]), bc.box.y / double(gd[1]), bc.box.z / double(gd[2])};
    auto rem = [](long a, long m) { long r = a % m; return r < 0 ? r + m : r; };
    long total = gd[0] * gd[1] * gd[2];
    std::vector<std::vector<int>> cells(total);
    for (int c = 0; c < ncg; ++c) {
        long cx = rem(long(std::floor(ref[c].x / cs[0])), gd[0]);
        long cy = rem(long(std::floor(ref[c].y / cs[1])), gd[1]);
        long cz = rem(long(std::floor(ref[c].z / cs[2])), gd[2]);
        cells[cx + cy * gd[0] + cz * gd[0] * gd[1]].push_back(c);
    }
    auto neighbors = [&](long cell) {
        long cx = cell % gd[0], cy = (cell / gd[0]) % gd[1], cz = cell / (gd[0] * gd[1]);
        std::set<long> s;
        for (long dx = -1; dx <= 1; ++dx)
            for (long dy = -1; dy <= 1; ++dy)
                for (long dz = -1; dz <= 1; ++dz)
                    s.insert(rem(cx + dx, gd[0]) + rem(cy + dy, gd[1]) * gd[0] +
                             rem(cz + dz, gd[2]) * gd[0] * gd[1]);
        return std::vector<long>(s.begin(), s.end());
    };
    int nth = nthreads > 1 ? nthreads : 1;
    std::vector<Lists> part(nth);
parallel_for(nth, size_t(total), [&](size_t cak, int tid) {
        long ca = long(cak);
        Lists& Lt = nth > 1 ? part[tid] : L;
        if (cells[ca].empty()) return;
        for (long cb : neighbors(ca)) {
            if (cb < ca || cells[cb].empty()) continue;
            if (ca == cb) {
                const auto& m = cells[ca];
                for (size_t i = 0; i < m.size(); ++i)
                    for (size_t j = i + 1; j < m.size(); ++j)
                        process_cg_pair(m[i], m[j], T, bc, pos, cog, c2s, c2l, Lt);
            } else {
                for (int c1 : cells[ca])
                    for (int c2 : cells[cb]) process_cg_pair(c1, c2, T, bc, pos, cog, c2s, c2l, Lt);
            }
        }
    });
    if (nth > 1)
        for (auto& p : part)
            for (int k = 0; k < 4; ++k) L.l[k].insert(L.l[k].end(), p.l[k].begin(), p.l[k].end());
}

struct CGPairGroup {
    int32_t ref_i, ref_j, start, end;
};  // params.rs:144-154

// Shared virial accumulation: virial[a][b] += r[a] * force[b]
inline void add_virial(Storage& s, V3 r, V3 f) {
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) s.vir[a][b] += comp(r, a) * comp(f, b);
}

struct Ctx {
    const Topo& T;
    const Boundary& bc;
    const CRF& crf;
    double fpe;
    const V3* pos;
};

// process_pairs (innerloops.rs:169-210): per-atom nearest image.
void process_pairs(const Ctx& C, const Pair* pairs, size_t n, bool virial, Storage& s) {
    for (size_t k = 0; k < n; ++k) {
        int i = pairs[k].first, j = pairs[k].second;
        V3 r = C.bc.nearest_image(C.pos[i], C.pos[j]);
        const LJ& lj = C.T.ljp(C.T.t->iac[i], C.T.t->iac[j]);
        double q = C.T.t->charge[i] * C.T.t->charge[j] * C.fpe;
        double fm, el, ec;
        lj_crf_interaction(r, lj.c6, lj.c12, q, C.crf, fm, el, ec);
        V3 f = r * fm;
        s.f[i] = s.f[i] + f;
        s.f[j] = s.f[j] - f;
        s.e_lj += el;
        s.e_crf += ec;
        s.group_add(C.T.egroup[i], C.T.egroup[j], el, ec);
        if (virial) add_virial(s, r, f);
    }
}

// process_pairs_cg_grouped (innerloops.rs:105-162): one image per CG pair.
void process_pairs_cg_grouped(const Ctx& C, const Pair* pairs, const CGPairGroup* groups,
                              size_t ng, bool virial, Storage& s) {
    for (size_t g = 0; g < ng; ++g) {
        V3 ri = C.pos[groups[g].ref_i], rj = C.pos[groups[g].ref_j];
        V3 rr = C.bc.nearest_image(ri, rj);
        double tx = rr.x - ri.x + rj.x, ty = rr.y - ri.y + rj.y, tz = rr.z - ri.z + rj.z;
        for (int k = groups[g].start; k < groups[g].end; ++k) {
            int i = pairs[k].first, j = pairs[k].second;
            V3 r{C.pos[i].x + tx - C.pos[j].x, C.pos[i].y + ty - C.pos[j].y,
                 C.pos[i].z + tz - C.pos[j].z};
            const LJ& lj = C.T.ljp(C.T.t->iac[i], C.T.t->iac[j]);
            double q = C.T.t->charge[i] * C.T.t->charge[j] * C.fpe;
            double fm, el, ec;
            lj_crf_interaction(r, lj.c6, lj.c12, q, C.crf, fm, el, ec);
            V3 f = r * fm;
            s.f[i] = s.f[i] + f;
            s.f[j] = s.f[j] - f;
            s.e_lj += el;
            s.e_crf += ec;
            s.group_add(C.T.egroup[i], C.T.egroup[j], el, ec);
            if (virial) add_virial(s, r, f);
        }
    }
}

// process_solvent_pairs (innerloops.rs:218-309): sentinel first-atom pairs,
// shared first-atom shift, parameter table taken from the first molecule.
void process_solvent_pairs(const Ctx& C, const Pair* pairs, size_t np, const Pair* first_of_list,
                           int nps, bool virial, Storage& s) {
    if (np == 0) return;
    int first_mol = first_of_list->first;
    double c6[4][4], c12[4][4], qq[4][4];
    for (int ai = 0; ai < nps; ++ai) {
        int ti = C.T.t->iac[first_mol + ai];
        double qi = C.T.t->charge[first_mol + ai];
        for (int aj = 0; aj < nps; ++aj) {
            const LJ& lj = C.T.ljp(ti, C.T.t->iac[first_mol + aj]);
            c6[ai][aj] = lj.c6;
            c12[ai][aj] = lj.c12;
            qq[ai][aj] = qi * C.T.t->charge[first_mol + aj] * C.fpe;
        }
    }
    for (size_t k = 0; k < np; ++k) {
        int i0 = pairs[k].first, j0 = pairs[k].second;
        V3 pi0 = C.pos[i0], pj0 = C.pos[j0];
        V3 rf = C.bc.nearest_image(pi0, pj0);
        double tx = rf.x - pi0.x + pj0.x, ty = rf.y - pi0.y + pj0.y, tz = rf.z - pi0.z + pj0.z;
        for (int ai = 0; ai < nps; ++ai) {
            int i = i0 + ai;
            double xi = C.pos[i].x + tx, yi = C.pos[i].y + ty, zi = C.pos[i].z + tz;
            for (int aj = 0; aj < nps; ++aj) {
                int j = j0 + aj;
                V3 r{xi - C.pos[j].x, yi - C.pos[j].y, zi - C.pos[j].z};
                double fm, el, ec;
                lj_crf_interaction(r, c6[ai][aj], c12[ai][aj], qq[ai][aj], C.crf, fm, el, ec);
                V3 f = r * fm;
                s.f[i] = s.f[i] + f;
                s.f[j] = s.f[j] - f;
                s.e_lj += el;
                s.e_crf += ec;
                s.group_add(C.T.egroup[i], C.T.egroup[j], el, ec);
                if (virial) add_virial(s, r, f);
            }
        }
    }
}

// Runs a loop body over [0, n) either serially into `dst` (reference order)
// or as a threaded fold/reduce with per-thread storages, mirroring rayon's
// par_chunks + ForceStorage::merge (innerloops.rs:640-665).
template <class F>
void fold_reduce(int nthreads, size_t n, size_t chunk, int natoms, int G, Storage& dst, F body) {
    if (nthreads <= 1 || n < 2 * chunk) {
        body(size_t(0), n, dst);
        return;
    }
    std::vector<Storage> part(nthreads);
    for (auto& p : part) p.init(natoms, G);
    size_t nchunks = (n + chunk - 1) / chunk;
parallel_for(nthreads, nchunks, [&](size_t c, int tid) {
        size_t b = c * chunk, e = std::min(n, b + chunk);
        body(b, e, part[tid]);
    });
    for (auto& p : part) dst.merge(p);
}

// rf_excluded_interactions (crates/gromos-forces/src/nonbonded/excluded.rs:25-112).
void rf_excluded(const Ctx& C, Storage& s) {
    const orc_topology* t = C.T.t;
    for (int i = 0; i < t->n_solute_atoms; ++i) {
        double term = -0.5 * t->charge[i] * t->charge[i] * C.fpe * C.crf.crf_cut;
        s.e_crf += term;
        s.group_add(C.T.egroup[i], C.T.egroup[i], 0.0, term);
        for (int k = t->excl_off[i]; k < t->excl_off[i + 1]; ++k) {
            int j = t->excl[k];
            if (j <= i) continue;
            V3 r = C.bc.nearest_image(C.pos[i], C.pos[j]);
            double r2 = len2(r);
            double q = t->charge[i] * t->charge[j] * C.fpe;
            double e = q * (-C.crf.crf_2cut3i * r2 - C.crf.crf_cut);
            s.e_crf += e;
            s.group_add(C.T.egroup[i], C.T.egroup[j], 0.0, e);
            V3 f = r * (q * C.crf.crf_cut3i);
            s.f[i] = s.f[i] + f;
            s.f[j] = s.f[j] - f;
            add_virial(s, r, f);
        }
    }
    for (int i = t->n_solute_atoms; i < t->n_atoms; ++i) {
        for (int k = t->excl_off[i]; k < t->excl_off[i + 1]; ++k) {
            int j = t->excl[k];
            if (j <= i) continue;
            V3 r = C.bc.nearest_image(C.pos[i], C.pos[j]);
            double r2 = len2(r);
            double e = -t->charge[i] * t->charge[j] * C.fpe * C.crf.crf_2cut3i * r2;
            s.e_crf += e;
            s.group_add(C.T.egroup[i], C.T.egroup[j], 0.0, e);
        }
    }
}

// one_four_interaction_loop (excluded.rs:131-206), coulomb_scaling = 1.
void one_four(const Ctx& C, Storage& s, double cscale) {
    const orc_topology* t = C.T.t;
    double el14 = 0, ec14 = 0;
    int nrow = t->n_atoms;
    for (int i = 0; i < nrow; ++i) {
        for (int k = t->o14_off[i]; k < t->o14_off[i + 1]; ++k) {
            int j = t->o14[k];
            if (j <= i) continue;
            V3 r = C.bc.nearest_image(C.pos[i], C.pos[j]);
            double r2 = len2(r);
            if (r2 < 1e-10) continue;
            const LJ& lj = C.T.ljp(t->iac[i], t->iac[j]);
            double inv_r2 = 1.0 / r2, inv_r6 = inv_r2 * inv_r2 * inv_r2;
            double e_lj = (lj.cs12 * inv_r6 - lj.cs6) * inv_r6;
            double f_lj = (12.0 * lj.cs12 * inv_r6 - 6.0 * lj.cs6) * inv_r6 * inv_r2;
            double q = t->charge[i] * t->charge[j] * C.fpe;
            double inv_r = std::sqrt(inv_r2);
            double e_crf = q * (inv_r * cscale - C.crf.crf_2cut3i * r2 - C.crf.crf_cut);
            double f_crf = q * (inv_r * cscale * inv_r2 + C.crf.crf_cut3i);
            V3 f = r * (f_lj + f_crf);
            s.f[i] = s.f[i] + f;
            s.f[j] = s.f[j] - f;
            el14 += e_lj;
            ec14 += e_crf;
            s.group_add(C.T.egroup[i], C.T.egroup[j], e_lj, e_crf);
            add_virial(s, r, f);
        }
    }
    s.e_lj += el14;
    s.e_crf += ec14;
}

// perturbed_lj_crf_interaction (perturbed.rs:124-266).
void perturbed_interaction(V3 r, double a_c6, double a_c12, double b_c6, double b_c12, double a_q,
                           double b_q, double alpha_lj, double alpha_crf, const LambdaParams& lp,
                           const CRF& crf, double fpe, double out[5]) {
    double r2 = len2(r);
    if (r2 < 1e-10) {
        for (int k = 0; k < 5; ++k) out[k] = 0.0;
        return;
    }
    double r6 = r2 * r2 * r2;
    double r4 = r2 * r2;
    double a_c126 = std::fabs(a_c6) > 1e-10 ? a_c12 / a_c6 : 0.0;
    double b_c126 = std::fabs(b_c6) > 1e-10 ? b_c12 / b_c6 : 0.0;
    double a_dist2soft = r2 + alpha_crf * lp.b_crfs2;
    double a_distisoft = 1.0 / std::sqrt(a_dist2soft);
    double a_dist3isoft = a_distisoft / a_dist2soft;
    double a_dist6soft = r6 + alpha_lj * lp.b_ljs2 * a_c126;
    double a_dist6isoft = 1.0 / a_dist6soft;
    double b_dist2soft = r2 + alpha_crf * lp.a_crfs2;
    double b_distisoft = 1.0 / std::sqrt(b_dist2soft);
    double b_dist3isoft = b_distisoft / b_dist2soft;
    double b_dist6soft = r6 + alpha_lj * lp.a_ljs2 * b_c126;
    double b_dist6isoft = 1.0 / b_dist6soft;
    double cut2 = crf.cutoff_sq;
    double a_cut2soft = cut2 + alpha_crf * lp.b_crfs2;
    double b_cut2soft = cut2 + alpha_crf * lp.a_crfs2;
    double a_cut2soft3 = a_cut2soft * a_cut2soft * a_cut2soft;
    double b_cut2soft3 = b_cut2soft * b_cut2soft * b_cut2soft;
    double a_crf_2cut3i = crf.crf_2cut3i / std::sqrt(a_cut2soft3);
    double b_crf_2cut3i = crf.crf_2cut3i / std::sqrt(b_cut2soft3);
    double a_crf_cut3i = 2.0 * a_crf_2cut3i;
    double b_crf_cut3i = 2.0 * b_crf_2cut3i;
    double a_crf_pert = 3.0 * a_crf_2cut3i / a_cut2soft;
    double b_crf_pert = 3.0 * b_crf_2cut3i / b_cut2soft;
    double force = (lp.a_crf_n * a_q * (a_dist3isoft + a_crf_cut3i) +
                    lp.b_crf_n * b_q * (b_dist3isoft + b_crf_cut3i)) *
                   fpe;
    force += -6.0 *
             (lp.a_lj_n * a_c6 * a_dist6isoft * a_dist6isoft +
              lp.b_lj_n * b_c6 * b_dist6isoft * b_dist6isoft) *
             r4;
    force += 12.0 *
             (lp.a_lj_n * a_c12 * a_dist6isoft * a_dist6isoft * a_dist6isoft +
              lp.b_lj_n * b_c12 * b_dist6isoft * b_dist6isoft * b_dist6isoft) *
             r4;
    double a_e_lj = (a_c12 * a_dist6isoft - a_c6) * a_dist6isoft;
    double b_e_lj = (b_c12 * b_dist6isoft - b_c6) * b_dist6isoft;
    double crf_cut = crf.crf_cut;
    double a_e_crf = a_q * (a_distisoft - a_crf_2cut3i * r2 - crf_cut);
    double b_e_crf = b_q * (b_distisoft - b_crf_2cut3i * r2 - crf_cut);
    double e_lj = lp.a_lj_n * a_e_lj + lp.b_lj_n * b_e_lj;
    double e_crf = (lp.a_crf_n * a_e_crf + lp.b_crf_n * b_e_crf) * fpe;
    double de_lj = -2.0 * alpha_lj *
                       (lp.a_lj_n * lp.b_ljs * a_c126 * a_dist6isoft * a_dist6isoft *
                            (2.0 * a_c12 * a_dist6isoft - a_c6) -
                        lp.b_lj_n * lp.a_ljs * b_c126 * b_dist6isoft * b_dist6isoft *
                            (2.0 * b_c12 * b_dist6isoft - b_c6)) +
                   double(lp.n) * (lp.b_lj_n1 * b_e_lj - lp.a_lj_n1 * a_e_lj);
    double de_crf = -(lp.a_crf_n * a_q * lp.b_crfs * (a_dist3isoft - a_crf_pert * r2) -
                      lp.b_crf_n * b_q * lp.a_crfs * (b_dist3isoft - b_crf_pert * r2)) *
                        fpe * alpha_crf +
                    double(lp.n) * (lp.b_crf_n1 * b_e_crf - lp.a_crf_n1 * a_e_crf) * fpe;
    out[0] = force;
    out[1] = e_lj;
    out[2] = e_crf;
    out[3] = de_lj;
    out[4] = de_crf;
}

struct PertInfo {
    int a_iac = 0, b_iac = 0;
    double a_q = 0, b_q = 0, alj = 0, acrf = 0;
};

inline bool pinfo(const Topo& T, int a, PertInfo& p) {
    if (!T.perturbed(a)) return false;
    int k = T.t->pert_idx[a];
    p = {T.t->pert_a_iac[k], T.t->pert_b_iac[k], T.t->pert_a_q[k], T.t->pert_b_q[k],
         T.t->pert_alpha_lj[k], T.t->pert_alpha_crf[k]};
    return true;
}

struct PertCorr {
    std::vector<V3> f;
    double de_lj = 0, de_crf = 0, dhdl = 0;
};

// perturbed_pairlist_correction (perturbed.rs:309-386).
void pert_pairlist_correction(const Ctx& C, const LambdaParams& lp, const std::vector<Pair>& pl,
                              PertCorr& out, Storage& grp) {
    const orc_topology* t = C.T.t;
    for (const Pair& pr : pl) {
        int i = pr.first, j = pr.second;
        PertInfo pi, pj;
        if (!pinfo(C.T, i, pi)) continue;
        bool hj = pinfo(C.T, j, pj);
        int a_iac_i = pi.a_iac, b_iac_i = pi.b_iac;
        int a_iac_j = hj ? pj.a_iac : t->iac[j], b_iac_j = hj ? pj.b_iac : t->iac[j];
        double a_q_i = pi.a_q, b_q_i = pi.b_q;
        double a_q_j = hj ? pj.a_q : t->charge[j], b_q_j = hj ? pj.b_q : t->charge[j];
        const LJ& lja = C.T.ljp(a_iac_i, a_iac_j);
        const LJ& ljb = C.T.ljp(b_iac_i, b_iac_j);
        double a_q = a_q_i * a_q_j, b_q = b_q_i * b_q_j;
        double alj = hj ? (pi.alj + pj.alj) * 0.5 : pi.alj;
        double acrf = hj ? (pi.acrf + pj.acrf) * 0.5 : pi.acrf;
        V3 r = C.bc.nearest_image(C.pos[i], C.pos[j]);
        double fa, ela, eca;
        lj_crf_interaction(r, lja.c6, lja.c12, a_q * C.fpe, C.crf, fa, ela, eca);
        double o[5];
        perturbed_interaction(r, lja.c6, lja.c12, ljb.c6, ljb.c12, a_q, b_q, alj, acrf, lp, C.crf,
                              C.fpe, o);
        V3 df = r * (o[0] - fa);
        out.f[i] = out.f[i] + df;
        out.f[j] = out.f[j] - df;
        out.de_lj += o[1] - ela;
        out.de_crf += o[2] - eca;
        out.dhdl += o[3] + o[4];
        grp.group_add(C.T.egroup[i], C.T.egroup[j], o[1] - ela, o[2] - eca);
    }
}

// perturbed_self_energy_correction (perturbed.rs:395-425).
void pert_self_correction(const Ctx& C, const LambdaParams& lp, double& de, double& dhdl,
                          Storage& grp) {
    const orc_topology* t = C.T.t;
    double n = double(lp.n);
    for (int a = 0; a < t->n_atoms; ++a) {
        PertInfo p;
        if (!pinfo(C.T, a, p)) continue;
        double qa2 = p.a_q * p.a_q, qb2 = p.b_q * p.b_q;
        double e_rf = (-(lp.a_crf_n * qa2) - lp.b_crf_n * qb2 + qa2) * C.crf.crf_cut * C.fpe;
        de += 0.5 * e_rf;
        double de_rf = n * (lp.a_crf_n1 * qa2 - lp.b_crf_n1 * qb2) * C.crf.crf_cut * C.fpe;
        dhdl += 0.5 * de_rf;
        grp.group_add(C.T.egroup[a], C.T.egroup[a], 0.0, 0.5 * e_rf);
    }
}

// perturbed_excluded_correction (perturbed.rs:431-511).
void pert_excluded_correction(const Ctx& C, const LambdaParams& lp, PertCorr& out, Storage& grp) {
    const orc_topology* t = C.T.t;
    for (int i = 0; i < t->n_solute_atoms; ++i) {
        PertInfo pi;
        bool hi = pinfo(C.T, i, pi);
        for (int k = t->excl_off[i]; k < t->excl_off[i + 1]; ++k) {
            int j = t->excl[k];
            if (j <= i) continue;
            PertInfo pj;
            bool hj = pinfo(C.T, j, pj);
            if (!hi && !hj) continue;
            double a_q_i = hi ? pi.a_q : t->charge[i], b_q_i = hi ? pi.b_q : t->charge[i];
            double a_q_j = hj ? pj.a_q : t->charge[j], b_q_j = hj ? pj.b_q : t->charge[j];
            double acrf = (hi && hj) ? (pi.acrf + pj.acrf) * 0.5 : (hi ? pi.acrf : pj.acrf);
            V3 r = C.bc.nearest_image(C.pos[i], C.pos[j]);
            double r2 = len2(r);
            double a_q = a_q_i * a_q_j, b_q = b_q_i * b_q_j;
            double cut2 = C.crf.cutoff_sq;
            double a_cut2soft = cut2 + acrf * lp.b_crfs2;
            double b_cut2soft = cut2 + acrf * lp.a_crfs2;
            double a_crf_2cut3i = C.crf.crf_2cut3i * std::sqrt(powi(cut2 / a_cut2soft, 3));
            double b_crf_2cut3i = C.crf.crf_2cut3i * std::sqrt(powi(cut2 / b_cut2soft, 3));
            double a_crf_cut3i = 2.0 * a_crf_2cut3i, b_crf_cut3i = 2.0 * b_crf_2cut3i;
            double a_crf_pert = 3.0 * a_crf_2cut3i / a_cut2soft;
            double b_crf_pert = 3.0 * b_crf_2cut3i / b_cut2soft;
            double a_e_crf = a_q * (-a_crf_2cut3i * r2 - C.crf.crf_cut);
            double b_e_crf = b_q * (-b_crf_2cut3i * r2 - C.crf.crf_cut);
            double e_crf_p = (lp.a_crf_n * a_e_crf + lp.b_crf_n * b_e_crf) * C.fpe;
            double f_p = (lp.a_crf_n * a_q * a_crf_cut3i + lp.b_crf_n * b_q * b_crf_cut3i) * C.fpe;
            double e_crf_a = a_q * C.fpe * (-C.crf.crf_2cut3i * r2 - C.crf.crf_cut);
            double f_a = a_q * C.fpe * C.crf.crf_cut3i;
            double n_exp = double(lp.n);
            double de_crf = ((lp.a_crf_n * a_q * lp.b_crfs * a_crf_pert -
                              lp.b_crf_n * b_q * lp.a_crfs * b_crf_pert) *
                                 r2 * acrf +
                             n_exp * (lp.b_crf_n1 * b_e_crf - lp.a_crf_n1 * a_e_crf)) *
                            C.fpe;
            V3 df = r * (f_p - f_a);
            out.f[i] = out.f[i] + df;
            out.f[j] = out.f[j] - df;
            out.de_crf += e_crf_p - e_crf_a;
            out.dhdl += de_crf;
            grp.group_add(C.T.egroup[i], C.T.egroup[j], 0.0, e_crf_p - e_crf_a);
        }
    }
}

// perturbed_one_four_correction (perturbed.rs:517-605).
void pert_one_four_correction(const Ctx& C, const LambdaParams& lp, PertCorr& out, Storage& grp) {
    const orc_topology* t = C.T.t;
    for (int i = 0; i < t->n_atoms; ++i) {
        PertInfo pi;
        bool hi = pinfo(C.T, i, pi);
        for (int k = t->o14_off[i]; k < t->o14_off[i + 1]; ++k) {
            int j = t->o14[k];
            if (j <= i) continue;
            PertInfo pj;
            bool hj = pinfo(C.T, j, pj);
            if (!hi && !hj) continue;
            int a_iac_i = hi ? pi.a_iac : t->iac[i], b_iac_i = hi ? pi.b_iac : t->iac[i];
            int a_iac_j = hj ? pj.a_iac : t->iac[j], b_iac_j = hj ? pj.b_iac : t->iac[j];
            double a_q_i = hi ? pi.a_q : t->charge[i], b_q_i = hi ? pi.b_q : t->charge[i];
            double a_q_j = hj ? pj.a_q : t->charge[j], b_q_j = hj ? pj.b_q : t->charge[j];
            const LJ& lja = C.T.ljp(a_iac_i, a_iac_j);
            const LJ& ljb = C.T.ljp(b_iac_i, b_iac_j);
            double a_q = a_q_i * a_q_j, b_q = b_q_i * b_q_j;
            double alj = (hi && hj) ? (pi.alj + pj.alj) * 0.5 : (hi ? pi.alj : pj.alj);
            double acrf = (hi && hj) ? (pi.acrf + pj.acrf) * 0.5 : (hi ? pi.acrf : pj.acrf);
            V3 r = C.bc.nearest_image(C.pos[i], C.pos[j]);
            double r2 = len2(r);
            if (r2 < 1e-10) continue;
            double inv_r2 = 1.0 / r2, inv_r6 = inv_r2 * inv_r2 * inv_r2, inv_r = std::sqrt(inv_r2);
            double e_lj_a = (lja.cs12 * inv_r6 - lja.cs6) * inv_r6;
            double f_lj_a = (12.0 * lja.cs12 * inv_r6 - 6.0 * lja.cs6) * inv_r6 * inv_r2;
            double e_crf_a = a_q * C.fpe * (inv_r - C.crf.crf_2cut3i * r2 - C.crf.crf_cut);
            double f_crf_a = a_q * C.fpe * (inv_r * inv_r2 + C.crf.crf_cut3i);
            double o[5];
            perturbed_interaction(r, lja.cs6, lja.cs12, ljb.cs6, ljb.cs12, a_q, b_q, alj, acrf, lp,
                                  C.crf, C.fpe, o);
            V3 df = r * (o[0] - (f_lj_a + f_crf_a));
            out.f[i] = out.f[i] + df;
            out.f[j] = out.f[j] - df;
            out.de_lj += o[1] - e_lj_a;
            out.de_crf += o[2] - e_crf_a;
            out.dhdl += o[3] + o[4];
            grp.group_add(C.T.egroup[i], C.T.egroup[j], o[1] - e_lj_a, o[2] - e_crf_a);
        }
    }
}

// perturbed_atom_pair_correction (perturbed.rs:624-707).
void pert_atom_pair_correction(const Ctx& C, const LambdaParams& lp, PertCorr& out, Storage& grp) {
    const orc_topology* t = C.T.t;
    double n_exp = double(lp.n);
    for (int k = 0; k < t->n_pert_pairs; ++k) {
        int i = t->pp_i[k], j = t->pp_j[k];
        bool in14 = C.T.o14_contains(i, j) || C.T.o14_contains(j, i);
        if (!in14) continue;
        V3 r = C.bc.nearest_image(C.pos[i], C.pos[j]);
        double r2 = len2(r);
        if (r2 < 1e-10) continue;
        double inv_r2 = 1.0 / r2, inv_r6 = inv_r2 * inv_r2 * inv_r2, inv_r = std::sqrt(inv_r2);
        const LJ& lj = C.T.ljp(t->iac[i], t->iac[j]);
        double e_lj_reg = (lj.cs12 * inv_r6 - lj.cs6) * inv_r6;
        double f_lj_reg = (12.0 * lj.cs12 * inv_r6 - 6.0 * lj.cs6) * inv_r6 * inv_r2;
        double q = t->charge[i] * t->charge[j] * C.fpe;
        double e_crf_reg = q * (inv_r - C.crf.crf_2cut3i * r2 - C.crf.crf_cut);
        double f_crf_reg = q * (inv_r * inv_r2 + C.crf.crf_cut3i);
        auto lj_pair = [&](int type, double& e, double& f) {
            if (type == 0) {
                e = (lj.c12 * inv_r6 - lj.c6) * inv_r6;
                f = (12.0 * lj.c12 * inv_r6 - 6.0 * lj.c6) * inv_r6 * inv_r2;
            } else {
                e = (lj.cs12 * inv_r6 - lj.cs6) * inv_r6;
                f = (12.0 * lj.cs12 * inv_r6 - 6.0 * lj.cs6) * inv_r6 * inv_r2;
            }
        };
        double e_lj_a, f_lj_a, e_lj_b = 0, f_lj_b = 0;
        lj_pair(t->pp_a_type[k], e_lj_a, f_lj_a);
        bool hasb = t->pp_b_type[k] >= 0;
        if (hasb) lj_pair(t->pp_b_type[k], e_lj_b, f_lj_b);
        double e_crf_a = e_crf_reg, f_crf_a = f_crf_reg;
        double e_crf_b = hasb ? e_crf_reg : 0.0, f_crf_b = hasb ? f_crf_reg : 0.0;
        double e_lj_pert = lp.a_lj_n * e_lj_a + lp.b_lj_n * e_lj_b;
        double e_crf_pert = lp.a_crf_n * e_crf_a + lp.b_crf_n * e_crf_b;
        double f_lj_pert = lp.a_lj_n * f_lj_a + lp.b_lj_n * f_lj_b;
        double f_crf_pert = lp.a_crf_n * f_crf_a + lp.b_crf_n * f_crf_b;
        double de_lj = n_exp * (lp.b_lj_n1 * e_lj_b - lp.a_lj_n1 * e_lj_a);
        double de_crf = n_exp * (lp.b_crf_n1 * e_crf_b - lp.a_crf_n1 * e_crf_a);
        V3 df = r * ((f_lj_pert - f_lj_reg) + (f_crf_pert - f_crf_reg));
        out.f[i] = out.f[i] + df;
        out.f[j] = out.f[j] - df;
        out.de_lj += e_lj_pert - e_lj_reg;
        out.de_crf += e_crf_pert - e_crf_reg;
        out.dhdl += de_lj + de_crf;
        // forcefield.rs:1020-1028 adds only Δe_lj of this pass to the totals
        grp.group_add(C.T.egroup[i], C.T.egroup[j], e_lj_pert - e_lj_reg, 0.0);
    }
}

}  // namespace

struct orc_pairlist {
    Lists L;
};

struct orc_ff {
    Topo* T = nullptr;
    orc_params p{};
    Boundary bc;
    CRF crf{};
    Lists L;
    int steps_since_update = 0;
    std::vector<CGPairGroup> groups;
    bool lists_cached = false;
    bool twin = false, lr_computed = false;
    Storage nb, lr;
    std::vector<int> atom_to_cg;
};

static void build_lists(const Topo& T, const orc_params& p, const Boundary& bc, const V3* pos,
                        Lists& L) {
    L.clear();
    // PairlistAlgorithm::from_imd (pairlist.rs:815-825): 2 -> cell list; the
    // cell list falls back to standard for non-rectangular boxes (:520-532).
    if (p.algorithm == 2 && bc.type == 1)
        pairlist_cell(T, bc, pos, p.rcutp, p.rcutl, p.skin, p.nthreads, L);
    else
        pairlist_standard(T, bc, pos, p.rcutp, p.rcutl, p.skin, L);
}

extern "C" {

void orc_crf_params(double cutoff, double eps, double epsrf, double kappa, double out[4]) {
    CRF c = make_crf(cutoff, eps, epsrf, kappa);
    out[0] = c.crf_cut;
    out[1] = c.crf_2cut3i;
    out[2] = c.crf_cut3i;
    out[3] = c.cutoff_sq;
}

orc_pairlist* orc_pairlist_build(const orc_topology* t, const orc_params* p, const double* pos) {
    Topo T(t);
    Boundary bc;
    bc.set(p->boundary, p->box);
    auto* pl = new orc_pairlist;
    build_lists(T, *p, bc, reinterpret_cast<const V3*>(pos), pl->L);
    return pl;
}

int64_t orc_pairlist_size(const orc_pairlist* pl, int which) {
    return (which < 0 || which > 3) ? -1 : int64_t(pl->L.l[which].size());
}

void orc_pairlist_get(const orc_pairlist* pl, int which, int32_t* out) {
    const auto& v = pl->L.l[which];
    for (size_t k = 0; k < v.size(); ++k) {
        out[2 * k] = v[k].first;
        out[2 * k + 1] = v[k].second;
    }
}

void orc_pairlist_free(orc_pairlist* pl) { delete pl; }

orc_ff* orc_ff_create(const orc_topology* t, const orc_params* p, const double* pos) {
    auto* ff = new orc_ff;
    ff->T = new Topo(t);
    ff->p = *p;
    ff->bc.set(p->boundary, p->box);
    ff->crf = make_crf(p->rcutl, p->epsilon, p->epsrf, p->kappa);  // md.rs:815 cutoff = RCUTL
    ff->twin = p->rcutp < p->rcutl - 1e-10;                         // forcefield.rs:126
    int G = ff->T->G;
    ff->nb.init(t->n_atoms, G);
    ff->lr.init(t->n_atoms, G);
    ff->atom_to_cg.assign(t->n_atoms, 0);
    for (int c = 0; c < t->n_cg; ++c)
        for (int a = t->cg_offsets[c]; a < t->cg_offsets[c + 1]; ++a) ff->atom_to_cg[a] = c;
    // initial pairlist generation (md.rs:864-867), counter reset to 0
    build_lists(*ff->T, ff->p, ff->bc, reinterpret_cast<const V3*>(pos), ff->L);
    ff->steps_since_update = 0;
    return ff;
}

void orc_ff_set_box(orc_ff* ff, const double box[3]) {
    ff->bc.set(ff->p.boundary, box);
    for (int k = 0; k < 3; ++k) ff->p.box[k] = box[k];
}

void orc_ff_destroy(orc_ff* ff) {
    if (!ff) return;
    delete ff->T;
    delete ff;
}

// Forcefield::apply, nonbonded part (forcefield.rs:226-1020).
int orc_ff_apply(orc_ff* ff, const double* pos_in, orc_result* out) {
    const Topo& T = *ff->T;
    const orc_topology* t = T.t;
    const V3* pos = reinterpret_cast<const V3*>(pos_in);
    int n = t->n_atoms;
    int nth = ff->p.nthreads > 1 ? ff->p.nthreads : 1;
    // use_cg_grouped_solute (forcefield.rs:267-283)
    bool cg_grouped = t->n_cg > 0 && (ff->bc.type == 0 ||
                                      std::min(std::min(ff->bc.half.x, ff->bc.half.y),
                                               ff->bc.half.z) > ff->p.rcutl + ff->p.skin + 0.3);
    bool updated = ff->steps_since_update >= ff->p.nsnb;  // pairlist.rs:105-107
    if (updated) {
        build_lists(T, ff->p, ff->bc, pos, ff->L);
        ff->steps_since_update = 0;
    }
    ff->steps_since_update += 1;
    auto& ss = ff->L.l[0];
    if (updated || !ff->lists_cached) {  // forcefield.rs:310-355
        ff->groups.clear();
        if (cg_grouped && !ss.empty()) {
            int start = 0;
            int ci = ff->atom_to_cg[ss[0].first], cj = ff->atom_to_cg[ss[0].second];
            for (size_t k = 1; k < ss.size(); ++k) {
                int a = ff->atom_to_cg[ss[k].first], b = ff->atom_to_cg[ss[k].second];
                if (a != ci || b != cj) {
                    ff->groups.push_back({t->cg_offsets[ci], t->cg_offsets[cj], start, int(k)});
                    start = int(k);
                    ci = a;
                    cj = b;
                }
            }
            ff->groups.push_back({t->cg_offsets[ci], t->cg_offsets[cj], start, int(ss.size())});
        }
        ff->lists_cached = true;
    }
    Storage& nb = ff->nb;
    nb.clear();
    Ctx C{T, ff->bc, ff->crf, ff->p.four_pi_eps_i, pos};
    bool vir = ff->p.virial != 0;
    int G = T.G;
    // short-range solute (forcefield.rs:417-547)
    if (cg_grouped) {
        const auto& gr = ff->groups;
        fold_reduce(nth, gr.size(), std::max<size_t>(1, gr.size() / nth + 1), n, G, nb,
                    [&](size_t b, size_t e, Storage& s) {
                        process_pairs_cg_grouped(C, ss.data(), gr.data() + b, e - b, vir, s);
                    });
    } else {
        fold_reduce(nth, ss.size(), 1024, n, G, nb, [&](size_t b, size_t e, Storage& s) {
            process_pairs(C, ss.data() + b, e - b, vir, s);
        });
    }
    // short-range solvent (forcefield.rs:549-618), par_chunks(512)
    const auto& vs = ff->L.l[2];
    if (!vs.empty())
        fold_reduce(nth, vs.size(), 512, n, G, nb, [&](size_t b, size_t e, Storage& s) {
            process_solvent_pairs(C, vs.data() + b, e - b, vs.data(), t->atoms_per_solvent, vir,
                                  s);
        });
    // twin range (forcefield.rs:620-727)
    if (ff->twin) {
        if (updated || !ff->lr_computed) {
            Storage& lr = ff->lr;
            lr.clear();
            for (int k : {1, 3}) {
                const auto& lst = ff->L.l[k];
                fold_reduce(nth, lst.size(), 1024, n, G, lr, [&](size_t b, size_t e, Storage& s) {
                    process_pairs(C, lst.data() + b, e - b, true, s);
                });
            }
            ff->lr_computed = true;
        }
        nb.merge(ff->lr);
    } else {
        if (!ff->L.l[1].empty()) process_pairs(C, ff->L.l[1].data(), ff->L.l[1].size(), true, nb);
        if (!ff->L.l[3].empty())
            process_solvent_pairs(C, ff->L.l[3].data(), ff->L.l[3].size(), ff->L.l[3].data(),
                                  t->atoms_per_solvent, true, nb);
    }
    rf_excluded(C, nb);
    if (T.has_o14) one_four(C, nb, 1.0);
    double dhdl = 0.0;
    bool anyp = false;
    if (t->pert_idx)
        for (int a = 0; a < n && !anyp; ++a) anyp = t->pert_idx[a] >= 0;
    if (anyp) {  // forcefield.rs:758-951
        double lam = ff->p.lambda;
        LambdaParams lp = from_lambda(lam, lam, lam, lam, 1.0, 1.0, 1.0, 1.0, ff->p.nlam);
        for (int k : {0, 1, 2, 3}) {
            const auto& lst = ff->L.l[k];
            if (lst.empty()) continue;
            PertCorr pc;
            pc.f.assign(n, V3{0, 0, 0});
            pert_pairlist_correction(C, lp, lst, pc, nb);
            nb.e_lj += pc.de_lj;
            nb.e_crf += pc.de_crf;
            dhdl += pc.dhdl;
            for (int a = 0; a < n; ++a) nb.f[a] = nb.f[a] + pc.f[a];
        }
        double de_self = 0, dh_self = 0;
        pert_self_correction(C, lp, de_self, dh_self, nb);
        nb.e_crf += de_self;
        dhdl += dh_self;
        {
            PertCorr pc;
            pc.f.assign(n, V3{0, 0, 0});
            pert_excluded_correction(C, lp, pc, nb);
            nb.e_crf += pc.de_crf;
            dhdl += pc.dhdl;
            for (int a = 0; a < n; ++a) nb.f[a] = nb.f[a] + pc.f[a];
        }
        if (T.has_o14) {
            PertCorr pc;
            pc.f.assign(n, V3{0, 0, 0});
            pert_one_four_correction(C, lp, pc, nb);
            nb.e_lj += pc.de_lj;
            nb.e_crf += pc.de_crf;
            dhdl += pc.dhdl;
            for (int a = 0; a < n; ++a) nb.f[a] = nb.f[a] + pc.f[a];
        }
        if (t->n_pert_pairs > 0) {
            PertCorr pc;
            pc.f.assign(n, V3{0, 0, 0});
            pert_atom_pair_correction(C, lp, pc, nb);
            nb.e_lj += pc.de_lj;
            dhdl += pc.dhdl;
            for (int a = 0; a < n; ++a) nb.f[a] = nb.f[a] + pc.f[a];
        }
    }
    out->e_lj = nb.e_lj;
    out->e_crf = nb.e_crf;
    out->dhdl = dhdl;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) out->virial[a * 3 + b] = nb.vir[a][b];
    if (out->forces)
        for (int a = 0; a < n; ++a) {
            out->forces[3 * a] = nb.f[a].x;
            out->forces[3 * a + 1] = nb.f[a].y;
            out->forces[3 * a + 2] = nb.f[a].z;
        }
    if (out->egroup_lj)
        std::memcpy(out->egroup_lj, nb.g_lj.data(), sizeof(double) * G * G);
    if (out->egroup_crf)
        std::memcpy(out->egroup_crf, nb.g_crf.data(), sizeof(double) * G * G);
    return 0;
}

void orc_lambda_params(double lj, double ljs, double crf, double crfs, double dlj, double dljs,
                       double dcrf, double dcrfs, int n, double out[17]) {
    LambdaParams p = from_lambda(lj, ljs, crf, crfs, dlj, dljs, dcrf, dcrfs, n);
    double v[17] = {p.a_lj_n,  p.b_lj_n,  p.a_crf_n, p.b_crf_n,  p.a_lj_n1, p.b_lj_n1,
                    p.a_crf_n1, p.b_crf_n1, p.a_ljs,  p.b_ljs,   p.a_ljs2, p.b_ljs2,
                    p.a_crfs,  p.b_crfs,  p.a_crfs2, p.b_crfs2, double(p.n)};
    std::memcpy(out, v, sizeof(v));
}

void orc_perturbed_pair(const double r[3], double a_c6, double a_c12, double b_c6, double b_c12,
                        double a_q, double b_q, double alpha_lj, double alpha_crf,
                        const double lp17[17], const double crf4[4], double fpe, double out[5]) {
    LambdaParams lp{lp17[0],  lp17[1],  lp17[2],  lp17[3],  lp17[4],  lp17[5],
                    lp17[6],  lp17[7],  lp17[8],  lp17[9],  lp17[10], lp17[11],
                    lp17[12], lp17[13], lp17[14], lp17[15], int(lp17[16])};
    CRF c{crf4[0], crf4[1], crf4[2], crf4[3]};
    perturbed_interaction(V3{r[0], r[1], r[2]}, a_c6, a_c12, b_c6, b_c12, a_q, b_q, alpha_lj,
                          alpha_crf, lp, c, fpe, out);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// MD step around Forcefield::apply, the sequence of gromos-md/src/bin/md.rs
// (:1144-1230) without thermostat: forces at r(t); leap-frog velocity
// v(t+dt/2) = v(t-dt/2) + F/m dt (leap_frog.rs:37-85); leap-frog position
// r(t+dt) = r(t) + v dt (leap_frog.rs:116-148); SETTLE of every solvent
// molecule (crates/gromos-integrators/src/constraints.rs:815-1010).
namespace {
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double vlen(V3 a) { return std::sqrt(dot(a, a)); }

// SETTLE (Miyamoto & Kollman 1992) for one molecule, following
// constraints.rs:857-975: canonical triangle, frame from the old plane and the
// new centre of mass, sin(phi), sin(psi), sin(theta), back-rotation.
// Returns false when one of the sines leaves [-1, 1] (the molecule is then
// left as the position update put it, as the reference does).
bool settle_one(const V3 old[3], V3 nw[3], V3 vel[3], double m_o, double m_h, double ra, double rb, double rc,
                double dt_i) {
    V3 b0 = old[1] - old[0], c0 = old[2] - old[0];
    const double mt = m_o + m_h + m_h;
    V3 d0 = (nw[0] * m_o + nw[1] * m_h + nw[2] * m_h) * (1.0 / mt);
    V3 a1 = nw[0] - d0, b1 = nw[1] - d0, c1 = nw[2] - d0;
    V3 n0 = cross(b0, c0);
    V3 n1 = cross(a1, n0);
    V3 n2 = cross(n0, n1);
    n0 = n0 * (1.0 / vlen(n0));
    n1 = n1 * (1.0 / vlen(n1));
    n2 = n2 * (1.0 / vlen(n2));
    V3 m1 = {n1.x, n2.x, n0.x}, m2 = {n1.y, n2.y, n0.y}, m0 = {n1.z, n2.z, n0.z};
    b0 = {dot(n1, b0), dot(n2, b0), dot(n0, b0)};
    c0 = {dot(n1, c0), dot(n2, c0), dot(n0, c0)};
    a1 = {dot(n1, a1), dot(n2, a1), dot(n0, a1)};
    b1 = {dot(n1, b1), dot(n2, b1), dot(n0, b1)};
    c1 = {dot(n1, c1), dot(n2, c1), dot(n0, c1)};
    const double sinphi = a1.z / ra;
    const double omp = 1.0 - sinphi * sinphi;
    if (omp < 0.0) return false;
    const double cosphi = std::sqrt(omp);
    const double sinpsi = (b1.z - c1.z) / (2.0 * rc * cosphi);
    const double omq = 1.0 - sinpsi * sinpsi;
    if (omq < 0.0) return false;
    const double cospsi = std::sqrt(omq);
    const double y_a2 = ra * cosphi, x_b2 = -rc * cospsi;
    const double y_b2 = -rb * cosphi - rc * sinpsi * sinphi, y_c2 = -rb * cosphi + rc * sinpsi * sinphi;
    const double alpha = x_b2 * (b0.x - c0.x) + b0.y * y_b2 + c0.y * y_c2;
    const double beta = x_b2 * (c0.y - b0.y) + b0.x * y_b2 + c0.x * y_c2;
    const double gamma = b0.x * b1.y - b1.x * b0.y + c0.x * c1.y - c1.x * c0.y;
    const double ab2 = alpha * alpha + beta * beta;
    const double sintheta = (alpha * gamma - beta * std::sqrt(ab2 - gamma * gamma)) / ab2;
    const double omt = 1.0 - sintheta * sintheta;
    if (omt < 0.0) return false;
    const double costheta = std::sqrt(omt);
    const V3 a3 = {-y_a2 * sintheta, y_a2 * costheta, a1.z};
    const V3 b3 = {x_b2 * costheta - y_b2 * sintheta, x_b2 * sintheta + y_b2 * costheta, b1.z};
    const V3 c3 = {-x_b2 * costheta - y_c2 * sintheta, -x_b2 * sintheta + y_c2 * costheta, c1.z};
    const V3 p[3] = {V3{dot(a3, m1), dot(a3, m2), dot(a3, m0)} + d0, V3{dot(b3, m1), dot(b3, m2), dot(b3, m0)} + d0,
                     V3{dot(c3, m1), dot(c3, m2), dot(c3, m0)} + d0};
    for (int k = 0; k < 3; ++k) {
        const V3 d = p[k] - nw[k];
        nw[k] = p[k];
        vel[k] = vel[k] + d * dt_i;
    }
    return true;
}
}  // namespace

extern "C" int orc_md_run(orc_ff* ff, double* pos_io, double* vel_io, const double* mass,
                          const orc_md_params* mp, int n_steps, double* e_kin, double energies[2]) {
    const orc_topology* t = ff->T->t;
    const int n = t->n_atoms, nsa = t->n_solute_atoms, aps = t->atoms_per_solvent;
    V3* pos = reinterpret_cast<V3*>(pos_io);
    V3* vel = reinterpret_cast<V3*>(vel_io);
    std::vector<double> f(size_t(n) * 3);
    std::vector<V3> old(n);
    const double dt = mp->dt;
    int failures = 0;
    double m_o = 0, m_h = 0, ra = 0, rb = 0, rc = 0;
    const bool settle = mp->settle && aps == 3 && n > nsa;
    if (settle) {  // canonical triangle (constraints.rs:836-840)
        m_o = mass[nsa];
        m_h = mass[nsa + 1];
        const double half_mo_div_mh = 0.5 * m_o / m_h;
        rc = 0.5 * mp->dist_hh;
        ra = std::sqrt(mp->dist_oh * mp->dist_oh - rc * rc) / (1.0 + half_mo_div_mh);
        rb = half_mo_div_mh * ra;
    }
    auto kinetic = [&]() {
        double ke = 0.0;
        for (int i = 0; i < n; ++i) ke += 0.5 * mass[i] * dot(vel[i], vel[i]);
        return ke;
    };
    // degrees of freedom: 3N minus the solvent constraints (md.rs:1158-1172, NDFMIN 0)
    const double dof = 3.0 * n - (settle ? 3.0 * ((n - nsa) / 3) : 0.0);
    double ke_in = kinetic();
    for (int step = 0; step < n_steps; ++step) {
        orc_result r{};
        r.forces = f.data();
        orc_ff_apply(ff, pos_io, &r);
        if (energies) {
            energies[0] = r.e_lj;
            energies[1] = r.e_crf;
        }
        double lambda = 1.0;
        if (mp->tau >= 0.0) {  // berendsen_thermostat.rs:74-98
            const double kB = 0.00831446261815324;
            double t = dof > 0.0 ? 2.0 * ke_in / (dof * kB) : 0.0;
            if (t < 1e-10) t = mp->temperature;
            if (t >= 1e-10)
                lambda = mp->tau == 0.0 ? std::sqrt(mp->temperature / t)
                                        : std::sqrt(1.0 + dt / mp->tau * (mp->temperature / t - 1.0));
        }
        for (int i = 0; i < n; ++i) {
            const V3 F = {f[3 * i], f[3 * i + 1], f[3 * i + 2]};
            vel[i] = (vel[i] + F * (1.0 / mass[i]) * dt) * lambda;
            old[i] = pos[i];
            pos[i] = pos[i] + vel[i] * dt;
        }
        if (settle)
            for (int i = nsa; i + 3 <= n; i += 3)
                if (!settle_one(&old[i], &pos[i], &vel[i], m_o, m_h, ra, rb, rc, 1.0 / dt)) ++failures;
        ke_in = kinetic();
    }
    if (e_kin) *e_kin = ke_in;
    return failures;
}
