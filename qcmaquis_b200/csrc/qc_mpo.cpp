// Exact QC Hamiltonian MPO (TwoU1) and its two-site fusion (host side, input prep).
//
// The reference builds its MPO term by term (models/chem/2u1/model.hpp:184-...,
// generate_mpo/tagged_mpo_maker_optim.hpp:212-...).  This builder is our own:
// every normal-ordered operator string of
//     H = sum h_pq a+_ps a_qs + 1/2 sum (pq|rs) a+_ps a+_rt a_st a_qs
// is written in Jordan-Wigner form (modes ordered site-major, up before
// down; the local operators are the reference's create/destroy/fill ops,
// model.hpp:57-91) and threaded through a finite-state automaton whose bond
// states are: V (nothing placed yet), D (term complete), L(prefix) = the
// operators already placed on the left (coefficient not yet applied) and
// R(suffix) = the operators still to come on the right (coefficient applied).
// A term is in an L state while fewer of its sites lie left of the bond than
// right of it, in an R state while more do, and on ties the smaller side
// holds the operators.  The integral coefficient is applied on the single
// transition from {V, L} to {R, D}; those entries are summed over terms,
// which yields the complementary-operator structure with O(L^2) bond
// dimension.  Any exact MPO of the same H gives the same energies; the
// contraction schedule is derived from whichever MPO is used.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <unordered_map>

#include "mpo.hpp"

namespace qcm {

void MPOTensor::finalize() {
    tables_.reset();
    row_ptr.assign(rows + 1, 0);
    for (auto r : b1) row_ptr[r + 1]++;
    for (uint32_t r = 0; r < rows; ++r) row_ptr[r + 1] += row_ptr[r];
    col_ptr.assign(cols + 1, 0);
    for (auto c : b2) col_ptr[c + 1]++;
    for (uint32_t c = 0; c < cols; ++c) col_ptr[c + 1] += col_ptr[c];
    col_ent.assign(b1.size(), 0);
    std::vector<uint32_t> fill(col_ptr.begin(), col_ptr.end() - 1);
    for (uint32_t e = 0; e < b1.size(); ++e) col_ent[fill[b2[e]]++] = e;  // increasing b1 within column
    if (herm_left.empty()) { herm_left.assign(rows, -1); phase_left.assign(rows, 1); }
    if (herm_right.empty()) { herm_right.assign(cols, -1); phase_right.assign(cols, 1); }
}

namespace {

using Mat4 = std::array<double, 16>;  // [out * 4 + in], states in qc_site_index() order

Mat4 mzero() { Mat4 m; m.fill(0.0); return m; }
Mat4 mul(const Mat4& A, const Mat4& B) {
    Mat4 C = mzero();
    for (int o = 0; o < 4; ++o)
        for (int k = 0; k < 4; ++k) {
            double a = A[o * 4 + k];
            if (a == 0.0) continue;
            for (int i = 0; i < 4; ++i) C[o * 4 + i] += a * B[k * 4 + i];
        }
    return C;
}

// states: 0 = |updown> (1,1), 1 = |up> (1,0), 2 = |down> (0,1), 3 = |0> (0,0)
struct LocalOps {
    Mat4 I, F, cdag[2], c[2];
    LocalOps() {
        I = mzero(); F = mzero();
        for (int s = 0; s < 4; ++s) I[s * 5] = 1.0;
        F[0] = 1.0; F[5] = -1.0; F[10] = -1.0; F[15] = 1.0;
        cdag[0] = mzero(); cdag[1] = mzero();
        cdag[0][1 * 4 + 3] = 1.0;   // |0>    -> |up>
        cdag[0][0 * 4 + 2] = 1.0;   // |down> -> |updown>
        cdag[1][2 * 4 + 3] = 1.0;   // |0>    -> |down>
        cdag[1][0 * 4 + 1] = -1.0;  // |up>   -> -|updown>  (up mode precedes down)
        for (int s = 0; s < 2; ++s) {
            c[s] = mzero();
            for (int o = 0; o < 4; ++o)
                for (int i = 0; i < 4; ++i) c[s][o * 4 + i] = cdag[s][i * 4 + o];
        }
    }
};

struct OpTable {
    std::vector<Mat4> mats;
    std::map<Mat4, uint32_t> ids;
    uint32_t raw(const Mat4& m) {
        auto it = ids.find(m);
        if (it != ids.end()) return it->second;
        uint32_t id = uint32_t(mats.size());
        mats.push_back(m);
        ids[m] = id;
        return id;
    }
    // normalises the sign (first non-zero entry positive); returns id and sign, or false if zero
    bool intern(const Mat4& m, uint32_t& id, double& sign) {
        int f = -1;
        for (int k = 0; k < 16; ++k) if (m[k] != 0.0) { f = k; break; }
        if (f < 0) return false;
        sign = m[f] > 0 ? 1.0 : -1.0;
        Mat4 n = m;
        if (sign < 0) for (auto& x : n) x = -x;
        id = raw(n);
        return true;
    }
};

enum : uint32_t { T_V = 0, T_L = 1, T_R = 2, T_D = 3 };

struct KeyInfo {
    uint32_t id;
    int edge;    // L: last site of prefix; R: first site of suffix
    int extent;  // L: max bond reached; R: min bond reached
    int parity;
};

inline uint64_t pack_pair(int site, uint32_t op) { return (uint64_t(site) << 16) | op; }

struct TKey {
    uint32_t in, out, op;
    bool operator==(const TKey& o) const { return in == o.in && out == o.out && op == o.op; }
};
struct TKeyHash {
    std::size_t operator()(const TKey& k) const {
        uint64_t h = (uint64_t(k.in) * 0x9E3779B97F4A7C15ull) ^ (uint64_t(k.out) * 0xC2B2AE3D27D4EB4Full) ^ k.op;
        return std::size_t(h ^ (h >> 29));
    }
};

struct Builder {
    int L;
    LocalOps lo;
    OpTable ops;
    uint32_t id_I, id_F;
    std::unordered_map<uint64_t, KeyInfo> Lkeys, Rkeys;
    std::vector<uint64_t> Lkey_of, Rkey_of;  // id -> packed key
    std::vector<std::unordered_map<TKey, double, TKeyHash>> trans;  // per site
    // integral provenance of the coefficient transitions (track): (integral id, factor) records
    bool track = false;
    using Prov = std::vector<std::pair<uint64_t, double>>;
    std::vector<std::unordered_map<TKey, Prov, TKeyHash>> ptrans;

    explicit Builder(int L_, bool track_ = false) : L(L_), trans(L_), track(track_), ptrans(track_ ? L_ : 0) {
        id_I = ops.raw(lo.I);
        id_F = ops.raw(lo.F);
    }

    uint32_t lkey(uint64_t key, int edge, int bond, int parity) {
        auto it = Lkeys.find(key);
        if (it == Lkeys.end()) {
            KeyInfo k{uint32_t(Lkey_of.size()), edge, bond, parity};
            Lkey_of.push_back(key);
            Lkeys.emplace(key, k);
            return k.id;
        }
        it->second.extent = std::max(it->second.extent, bond);
        return it->second.id;
    }
    uint32_t rkey(uint64_t key, int edge, int bond, int parity) {
        auto it = Rkeys.find(key);
        if (it == Rkeys.end()) {
            KeyInfo k{uint32_t(Rkey_of.size()), edge, bond, parity};
            Rkey_of.push_back(key);
            Rkeys.emplace(key, k);
            return k.id;
        }
        it->second.extent = std::min(it->second.extent, bond);
        return it->second.id;
    }

    // One term: product (left to right) of n fermion operators; its coefficient is
    // sum_j pv[j].second * x[pv[j].first] (npv records, recorded when tracking).
    void add_term(int n, const int* mode, const bool* dag, double coeff, const std::pair<uint64_t, double>* pv = nullptr,
                  int npv = 0) {
        int sites[4], ns = 0;
        for (int k = 0; k < n; ++k) {
            int s = mode[k] >> 1;
            bool seen = false;
            for (int j = 0; j < ns; ++j) seen |= (sites[j] == s);
            if (!seen) sites[ns++] = s;
        }
        std::sort(sites, sites + ns);
        uint32_t opid[4];
        int par[4];
        double sgn = 1.0;
        for (int j = 0; j < ns; ++j) {
            int x = sites[j];
            Mat4 M = lo.I;
            int cnt = 0;
            for (int k = 0; k < n; ++k) {
                int s = mode[k] >> 1, sp = mode[k] & 1;
                if (s == x) { M = mul(M, dag[k] ? lo.cdag[sp] : lo.c[sp]); ++cnt; }
                else if (s > x) M = mul(M, lo.F);
            }
            double sign;
            if (!ops.intern(M, opid[j], sign)) return;  // operator string vanishes
            coeff *= sign;
            sgn *= sign;
            par[j] = cnt & 1;
        }
        const int mid = (L - 2) / 2;  // ties: L state for bonds p <= mid, R state after
        auto type_at = [&](int p, int& nl) -> uint32_t {
            nl = 0;
            while (nl < ns && sites[nl] <= p) ++nl;
            int nr = ns - nl;
            if (nl == 0) return T_V;
            if (nr == 0) return T_D;
            if (nl < nr) return T_L;
            if (nl > nr) return T_R;
            return (p <= mid) ? T_L : T_R;
        };
        auto sym_at = [&](int p) -> uint32_t {
            int nl;
            uint32_t t = type_at(p, nl);
            if (t == T_V || t == T_D) return t << 28;
            if (t == T_L) {
                uint64_t key = uint64_t(nl) << 60;
                int parity = 0;
                for (int j = 0; j < nl; ++j) { key |= pack_pair(sites[j], opid[j]) << (30 * (1 - j)); parity ^= par[j]; }
                return (T_L << 28) | lkey(key, sites[nl - 1], p, parity);
            }
            uint64_t key = uint64_t(ns - nl) << 60;
            int parity = 0;
            for (int j = nl; j < ns; ++j) { key |= pack_pair(sites[j], opid[j]) << (30 * (1 - (j - nl))); parity ^= par[j]; }
            return (T_R << 28) | rkey(key, sites[nl], p, parity);
        };
        // event sites: term sites and the tie flip site (mid + 1)
        int ev[6], ne = 0;
        for (int j = 0; j < ns; ++j) ev[ne++] = sites[j];
        if (mid + 1 > sites[0] && mid + 1 < sites[ns - 1]) {
            bool is_site = false;
            for (int j = 0; j < ns; ++j) is_site |= (sites[j] == mid + 1);
            if (!is_site) ev[ne++] = mid + 1;
        }
        std::sort(ev, ev + ne);
        // walk the bonds between events so that every L/R key's extent is recorded
        for (int e = 0; e < ne; ++e) {
            int y = ev[e];
            uint32_t sin = sym_at(y - 1);
            uint32_t sout = sym_at(y);
            // extend the state of bond y up to the bond before the next event
            if (e + 1 < ne) sym_at(ev[e + 1] - 1);
            uint32_t op;
            int j = -1;
            for (int k = 0; k < ns; ++k) if (sites[k] == y) j = k;
            if (j >= 0) op = opid[j];
            else {
                int parity = 0;
                for (int k = 0; k < ns; ++k) if (sites[k] < y) parity ^= par[k];
                op = parity ? id_F : id_I;
            }
            uint32_t tin = sin >> 28, tout = sout >> 28;
            bool sw = (tin == T_V || tin == T_L) && (tout == T_R || tout == T_D);
            TKey key{sin, sout, op};
            if (sw) {
                trans[y][key] += coeff;
                if (track) {
                    Prov& pr = ptrans[y][key];
                    for (int k = 0; k < npv; ++k) pr.push_back({pv[k].first, pv[k].second * sgn});
                }
            } else trans[y].emplace(key, 1.0);
        }
    }

    // Hermitian conjugate of an interned local operator: the id of its normalised
    // transpose and the sign that normalisation took out (false: not in the table)
    bool conj_op(uint32_t id, uint32_t& cid, int& sign) const {
        const Mat4& M = ops.mats[id];
        Mat4 t;
        for (int o = 0; o < 4; ++o)
            for (int i = 0; i < 4; ++i) t[o * 4 + i] = M[i * 4 + o];
        int f = -1;
        for (int k = 0; k < 16; ++k) if (t[k] != 0.0) { f = k; break; }
        if (f < 0) return false;
        sign = t[f] > 0 ? 1 : -1;
        if (sign < 0) for (auto& x : t) x = -x;
        auto it = ops.ids.find(t);
        if (it == ops.ids.end()) return false;
        cid = it->second;
        return true;
    }

    // Conjugate of an L or R key: every (site, operator) pair replaced by the operator's
    // transpose.  The bond operator of the conjugate key is the adjoint of this key's up to
    // the product of the normalisation signs over the key's own sites, on both sides of the
    // bond (the coefficients of conjugate terms carry the same signs), which is the phase.
    bool conj_key(uint64_t key, uint64_t& ckey, int& phase) const {
        const uint64_t n = key >> 60;
        ckey = n << 60;
        phase = 1;
        for (uint64_t j = 0; j < n; ++j) {
            const int shift = int(30 * (1 - j));
            const uint64_t pr = (key >> shift) & ((uint64_t(1) << 30) - 1);
            uint32_t cid;
            int s;
            if (!conj_op(uint32_t(pr & 0xFFFF), cid, s)) return false;
            phase *= s;
            ckey |= ((pr & ~uint64_t(0xFFFF)) | cid) << shift;
        }
        return true;
    }

    MPO finish(double cutoff, IntegralProvenance* prov = nullptr) {
        // pass-through transitions of L and R keys over their extents
        for (auto& kv : Lkeys) {
            const KeyInfo& k = kv.second;
            for (int y = k.edge + 1; y <= k.extent; ++y)
                trans[y].emplace(TKey{(T_L << 28) | k.id, (T_L << 28) | k.id, k.parity ? id_F : id_I}, 1.0);
        }
        for (auto& kv : Rkeys) {
            const KeyInfo& k = kv.second;
            for (int y = k.extent + 1; y <= k.edge - 1; ++y)
                trans[y].emplace(TKey{(T_R << 28) | k.id, (T_R << 28) | k.id, k.parity ? id_F : id_I}, 1.0);
        }
        for (int y = 0; y <= L - 2; ++y) trans[y].emplace(TKey{T_V << 28, T_V << 28, id_I}, 1.0);
        for (int y = 1; y <= L - 1; ++y) trans[y].emplace(TKey{T_D << 28, T_D << 28, id_I}, 1.0);

        // bond numbering: bond p (between site p and p+1), p = -1 .. L-1
        std::vector<std::unordered_map<uint32_t, uint32_t>> bond(L + 1);
        std::vector<uint32_t> bdim(L + 1, 0);
        for (int p = -1; p <= L - 1; ++p) {
            auto& m = bond[p + 1];
            uint32_t n = 0;
            if (p <= L - 2) m[T_V << 28] = n++;
            std::vector<std::pair<uint64_t, uint32_t>> ls, rs;
            if (p >= 0 && p <= L - 2) {
                for (auto& kv : Lkeys) if (kv.second.edge <= p && p <= kv.second.extent) ls.push_back({kv.first, kv.second.id});
                for (auto& kv : Rkeys) if (kv.second.extent <= p && p <= kv.second.edge - 1) rs.push_back({kv.first, kv.second.id});
            }
            std::sort(ls.begin(), ls.end());
            std::sort(rs.begin(), rs.end());
            for (auto& e : ls) m[(T_L << 28) | e.second] = n++;
            for (auto& e : rs) m[(T_R << 28) | e.second] = n++;
            if (p >= 0) m[T_D << 28] = n++;
            bdim[p + 1] = n;
        }

        // Hermitian pairs per bond (the reference registers them in create_mpo,
        // tagged_mpo_maker_optim.hpp:292-307): an L or R key and its conjugate key are
        // partners, a key equal to its conjugate is self-adjoint; V and D, the keys
        // without operators, are left unregistered as the reference leaves its trivial keys
        std::vector<std::vector<int32_t>> bherm(L + 1), bphase(L + 1);
        for (int p = -1; p <= L - 1; ++p) {
            auto& m = bond[p + 1];
            auto& hv = bherm[p + 1];
            auto& ph = bphase[p + 1];
            hv.assign(bdim[p + 1], -1);
            ph.assign(bdim[p + 1], 1);
            for (auto& kv : m) {
                const uint32_t t = kv.first >> 28, id = kv.first & ((1u << 28) - 1);
                if (t != T_L && t != T_R) continue;
                const auto& keys = (t == T_L) ? Lkeys : Rkeys;
                const uint64_t key = (t == T_L) ? Lkey_of[id] : Rkey_of[id];
                uint64_t ckey;
                int phase;
                if (!conj_key(key, ckey, phase)) continue;
                auto ck = keys.find(ckey);
                if (ck == keys.end()) continue;
                auto cb = m.find((t << 28) | ck->second.id);
                if (cb == m.end()) continue;
                hv[kv.second] = int32_t(cb->second);
                ph[kv.second] = phase;
            }
        }

        auto sops = std::make_shared<std::vector<SparseOp>>();
        for (auto& M : ops.mats) {
            SparseOp s;
            for (int o = 0; o < 4; ++o)
                for (int i = 0; i < 4; ++i)
                    if (M[o * 4 + i] != 0.0) { s.in.push_back(i); s.out.push_back(o); s.val.push_back(M[o * 4 + i]); }
            sops->push_back(s);
        }

        MPO mpo;
        mpo.t.resize(L);
        if (prov) {
            prov->ptr.assign(L, {});
            prov->id.assign(L, {});
            prov->val.assign(L, {});
        }
        for (int y = 0; y < L; ++y) {
            MPOTensor& T = mpo.t[y];
            T.rows = bdim[y];
            T.cols = bdim[y + 1];
            T.ops = sops;
            T.phys = qc_site_index();
            struct E { uint32_t b1, b2, op; double v; const Prov* pv; };
            std::vector<E> es;
            for (auto& kv : trans[y]) {
                if (!track && std::fabs(kv.second) <= cutoff) continue;
                auto ib = bond[y].find(kv.first.in);
                auto ob = bond[y + 1].find(kv.first.out);
                if (ib == bond[y].end() || ob == bond[y + 1].end())
                    throw std::runtime_error("qc mpo: dangling automaton state");
                const Prov* pv = nullptr;
                if (track) {
                    auto it = ptrans[y].find(kv.first);
                    if (it != ptrans[y].end()) pv = &it->second;
                }
                es.push_back({ib->second, ob->second, kv.first.op, kv.second, pv});
            }
            std::sort(es.begin(), es.end(), [](const E& a, const E& b) {
                if (a.b1 != b.b1) return a.b1 < b.b1;
                if (a.b2 != b.b2) return a.b2 < b.b2;
                return a.op < b.op;
            });
            for (auto& e : es) { T.b1.push_back(e.b1); T.b2.push_back(e.b2); T.op.push_back(e.op); T.scale.push_back(e.v); }
            if (prov) {
                // per entry its records by integral id, duplicates summed
                auto& pp = prov->ptr[y];
                auto& pi = prov->id[y];
                auto& pw = prov->val[y];
                pp.assign(1, 0);
                Prov r;
                for (auto& e : es) {
                    r.clear();
                    if (e.pv) r = *e.pv;
                    std::sort(r.begin(), r.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
                    for (std::size_t k = 0; k < r.size();) {
                        const uint64_t id = r[k].first;
                        double f = 0.0;
                        for (; k < r.size() && r[k].first == id; ++k) f += r[k].second;
                        if (f != 0.0) { pi.push_back(id); pw.push_back(f); }
                    }
                    pp.push_back(pi.size());
                }
            }
            T.herm_left = bherm[y]; T.phase_left = bphase[y];
            T.herm_right = bherm[y + 1]; T.phase_right = bphase[y + 1];
            T.finalize();
        }
        return mpo;
    }
};

}  // namespace

MPO build_qc_mpo(int L, const double* h, const double* V, double cutoff, IntegralProvenance* prov) {
    if (L < 2) throw std::runtime_error("qc mpo: need at least two orbitals");
    Builder B(L, prov != nullptr);
    const uint64_t L2 = uint64_t(L) * L;
    const int M = 2 * L;
    auto Vat = [&](int p, int q, int r, int s) { return V[((std::size_t(p) * L + q) * L + r) * L + s]; };
    // one-electron part
    for (int p = 0; p < L; ++p)
        for (int q = 0; q < L; ++q) {
            double v = h[p * L + q];
            if (!prov && std::fabs(v) <= cutoff) continue;
            const std::pair<uint64_t, double> pv{uint64_t(p) * L + q, 1.0};
            for (int s = 0; s < 2; ++s) {
                int mode[2] = {2 * p + s, 2 * q + s};
                bool dag[2] = {true, false};
                B.add_term(2, mode, dag, v, &pv, 1);
            }
        }
    // two-electron part, one canonical string a+_A a+_B a_C a_D per A<B, C<D
    auto W = [&](int i, int j, int k, int l) -> double {
        if ((i & 1) != (l & 1) || (j & 1) != (k & 1)) return 0.0;
        return 0.5 * Vat(i >> 1, l >> 1, j >> 1, k >> 1);
    };
    // the provenance record of W(i, j, k, l) with sign f (none where the spins forbid it)
    auto Wp = [&](int i, int j, int k, int l, double f, std::pair<uint64_t, double>* pv, int& n) {
        if ((i & 1) != (l & 1) || (j & 1) != (k & 1)) return;
        const uint64_t p = uint64_t(i >> 1), q = uint64_t(l >> 1), r = uint64_t(j >> 1), t = uint64_t(k >> 1);
        pv[n++] = {L2 + ((p * L + q) * L + r) * L + t, 0.5 * f};
    };
    for (int A = 0; A < M; ++A)
        for (int Bm = A + 1; Bm < M; ++Bm)
            for (int C = 0; C < M; ++C)
                for (int D = C + 1; D < M; ++D) {
                    // spin conservation: spins of {A,B} equal spins of {C,D}
                    if (((A & 1) + (Bm & 1)) != ((C & 1) + (D & 1))) continue;
                    double g = W(A, Bm, C, D) - W(Bm, A, C, D) - W(A, Bm, D, C) + W(Bm, A, D, C);
                    std::pair<uint64_t, double> pv[4];
                    int npv = 0;
                    if (prov) {
                        Wp(A, Bm, C, D, 1.0, pv, npv);
                        Wp(Bm, A, C, D, -1.0, pv, npv);
                        Wp(A, Bm, D, C, -1.0, pv, npv);
                        Wp(Bm, A, D, C, 1.0, pv, npv);
                        if (!npv) continue;
                    } else if (std::fabs(g) <= cutoff) continue;
                    int mode[4] = {A, Bm, C, D};
                    bool dag[4] = {true, true, false, false};
                    B.add_term(4, mode, dag, g, pv, npv);
                }
    return B.finish(cutoff, prov);
}

void integral_gradient(const IntegralProvenance& prov, const std::vector<std::vector<double>>& grad, double* dx,
                       uint64_t n) {
    if (grad.size() != prov.ptr.size()) throw std::runtime_error("integral gradient: one gradient per site tensor");
    for (std::size_t k = 0; k < grad.size(); ++k) {
        const auto& pp = prov.ptr[k];
        if (grad[k].size() + 1 != pp.size()) throw std::runtime_error("integral gradient: entry count differs from the MPO's");
        for (std::size_t e = 0; e < grad[k].size(); ++e)
            for (uint64_t j = pp[e]; j < pp[e + 1]; ++j) {
                const uint64_t id = prov.id[k][j];
                if (id >= n) throw std::runtime_error("integral gradient: integral id out of range");
                dx[id] += prov.val[k][j] * grad[k][e];
            }
    }
}

// ---------------------------------------------------------------------------
// two-site MPO

MPO make_twosite_mpo(const MPO& m) {
    MPO out;
    out.twosite = true;
    std::size_t L = m.t.size();
    if (L < 2) return out;
    out.t.resize(L - 1);
    for (std::size_t p = 0; p + 1 < L; ++p) {
        const MPOTensor& W1 = m.t[p];
        const MPOTensor& W2 = m.t[p + 1];
        const Index& ph1 = W1.phys;
        const Index& ph2 = W2.phys;
        Index tw = index_product(ph1, ph2);
        ProductBasis pb(ph1, ph2);
        StateMap sm1(ph1), sm2(ph2), smt(tw);
        // (state1, state2) -> two-site state, sub-index pb(c1,c2) + ss1*d2 + ss2 (alps_detail op_kron)
        std::vector<uint32_t> tws(sm1.nstates() * sm2.nstates());
        for (int s1 = 0; s1 < sm1.nstates(); ++s1)
            for (int s2 = 0; s2 < sm2.nstates(); ++s2) {
                Charge c1 = ph1[sm1.sector[s1]].first, c2 = ph2[sm2.sector[s2]].first;
                std::size_t d2 = ph2[sm2.sector[s2]].second;
                std::size_t sec = tw.position(c1 + c2);
                tws[s1 * sm2.nstates() + s2] = uint32_t(smt.first[sec] + pb(c1, c2) + sm1.sub[s1] * d2 + sm2.sub[s2]);
            }
        const int n2 = sm2.nstates();
        auto kron = [&](const SparseOp& a, const SparseOp& b, double f, std::map<std::pair<uint32_t, uint32_t>, double>& acc) {
            for (std::size_t i = 0; i < a.val.size(); ++i)
                for (std::size_t j = 0; j < b.val.size(); ++j)
                    acc[{tws[a.in[i] * n2 + b.in[j]], tws[a.out[i] * n2 + b.out[j]]}] += f * a.val[i] * b.val[j];
        };
        auto sops = std::make_shared<std::vector<SparseOp>>();
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> kron_ids;
        auto to_sparse = [](const std::map<std::pair<uint32_t, uint32_t>, double>& acc) {
            SparseOp s;
            for (auto& kv : acc)
                if (kv.second != 0.0) { s.in.push_back(kv.first.first); s.out.push_back(kv.first.second); s.val.push_back(kv.second); }
            return s;
        };
        MPOTensor T;
        T.rows = W1.rows;
        T.cols = W2.cols;
        T.phys = tw;
        T.ops = sops;
        T.herm_left = W1.herm_left; T.phase_left = W1.phase_left;
        T.herm_right = W2.herm_right; T.phase_right = W2.phase_right;
        for (uint32_t b1 = 0; b1 < W1.rows; ++b1) {
            // b3 -> list of (entry1, entry2)
            std::map<uint32_t, std::vector<std::pair<uint32_t, uint32_t>>> sum;
            for (uint32_t e1 = W1.row_ptr[b1]; e1 < W1.row_ptr[b1 + 1]; ++e1) {
                uint32_t b2 = W1.b2[e1];
                for (uint32_t e2 = W2.row_ptr[b2]; e2 < W2.row_ptr[b2 + 1]; ++e2) sum[W2.b2[e2]].push_back({e1, e2});
            }
            for (auto& kv : sum) {
                uint32_t b3 = kv.first;
                auto& lst = kv.second;
                std::map<uint32_t, int> b2s;
                for (auto& pr : lst) b2s[W1.b2[pr.first]]++;
                if (lst.size() == 1) {
                    uint32_t e1 = lst[0].first, e2 = lst[0].second;
                    auto key = std::make_pair(W1.op[e1], W2.op[e2]);
                    auto it = kron_ids.find(key);
                    uint32_t id;
                    if (it == kron_ids.end()) {
                        std::map<std::pair<uint32_t, uint32_t>, double> acc;
                        kron((*W1.ops)[W1.op[e1]], (*W2.ops)[W2.op[e2]], 1.0, acc);
                        id = uint32_t(sops->size());
                        sops->push_back(to_sparse(acc));
                        kron_ids[key] = id;
                    } else id = it->second;
                    if ((*sops)[id].val.empty()) continue;
                    T.b1.push_back(b1); T.b2.push_back(b3); T.op.push_back(id);
                    T.scale.push_back(W1.scale[e1] * W2.scale[e2]);
                } else {
                    std::map<std::pair<uint32_t, uint32_t>, double> acc;
                    for (auto& pr : lst)
                        kron((*W1.ops)[W1.op[pr.first]], (*W2.ops)[W2.op[pr.second]],
                             W1.scale[pr.first] * W2.scale[pr.second], acc);
                    SparseOp s = to_sparse(acc);
                    if (s.val.empty()) continue;
                    uint32_t id = uint32_t(sops->size());
                    sops->push_back(std::move(s));
                    T.b1.push_back(b1); T.b2.push_back(b3); T.op.push_back(id); T.scale.push_back(1.0);
                }
            }
        }
        T.finalize();
        out.t[p] = std::move(T);
    }
    return out;
}

// ---------------------------------------------------------------------------
// binary interchange format (little endian):
//   "QMPO" u32 version=1 u32 ntensors u32 twosite
//   per tensor: u32 nsec, nsec x (i32 a, i32 b, u32 size); u32 rows, u32 cols, u64 nnz,
//     nnz x (u32 b1, u32 b2, u32 op, f64 scale); rows x (i32 herm, i32 phase);
//     cols x (i32 herm, i32 phase); u32 nops; per op: u32 n, n x (u32 in, u32 out, f64 val)

namespace {
struct Writer {
    std::vector<uint8_t> b;
    template <class T> void put(T v) { const uint8_t* p = reinterpret_cast<const uint8_t*>(&v); b.insert(b.end(), p, p + sizeof(T)); }
};
struct Reader {
    const uint8_t* p; std::size_t n, k = 0;
    template <class T> T get() {
        if (k + sizeof(T) > n) throw std::runtime_error("mpo blob truncated");
        T v; std::memcpy(&v, p + k, sizeof(T)); k += sizeof(T); return v;
    }
};
}  // namespace

std::vector<uint8_t> serialize_mpo(const MPO& m) {
    Writer w;
    w.put<uint32_t>(0x4F504D51u);  // "QMPO"
    w.put<uint32_t>(1);
    w.put<uint32_t>(uint32_t(m.t.size()));
    w.put<uint32_t>(m.twosite ? 1 : 0);
    for (auto& T : m.t) {
        w.put<uint32_t>(uint32_t(T.phys.size()));
        for (auto& s : T.phys.d) { w.put<int32_t>(s.first.a); w.put<int32_t>(s.first.b); w.put<uint32_t>(uint32_t(s.second)); }
        w.put<uint32_t>(T.rows); w.put<uint32_t>(T.cols); w.put<uint64_t>(T.b1.size());
        for (std::size_t e = 0; e < T.b1.size(); ++e) { w.put(T.b1[e]); w.put(T.b2[e]); w.put(T.op[e]); w.put(T.scale[e]); }
        for (uint32_t r = 0; r < T.rows; ++r) { w.put<int32_t>(T.herm_left[r]); w.put<int32_t>(T.phase_left[r]); }
        for (uint32_t c = 0; c < T.cols; ++c) { w.put<int32_t>(T.herm_right[c]); w.put<int32_t>(T.phase_right[c]); }
        w.put<uint32_t>(uint32_t(T.ops->size()));
        for (auto& o : *T.ops) {
            w.put<uint32_t>(uint32_t(o.val.size()));
            for (std::size_t i = 0; i < o.val.size(); ++i) { w.put(o.in[i]); w.put(o.out[i]); w.put(o.val[i]); }
        }
    }
    return w.b;
}

MPO deserialize_mpo(const uint8_t* p, std::size_t n) {
    Reader r{p, n};
    if (r.get<uint32_t>() != 0x4F504D51u) throw std::runtime_error("not an MPO blob");
    if (r.get<uint32_t>() != 1) throw std::runtime_error("unsupported MPO blob version");
    MPO m;
    uint32_t nt = r.get<uint32_t>();
    m.twosite = r.get<uint32_t>() != 0;
    m.t.resize(nt);
    for (auto& T : m.t) {
        uint32_t ns = r.get<uint32_t>();
        for (uint32_t s = 0; s < ns; ++s) {
            int a = r.get<int32_t>(), b = r.get<int32_t>();
            uint32_t sz = r.get<uint32_t>();
            T.phys.d.push_back({Charge(a, b), sz});
        }
        T.rows = r.get<uint32_t>(); T.cols = r.get<uint32_t>();
        uint64_t nnz = r.get<uint64_t>();
        T.b1.resize(nnz); T.b2.resize(nnz); T.op.resize(nnz); T.scale.resize(nnz);
        for (uint64_t e = 0; e < nnz; ++e) { T.b1[e] = r.get<uint32_t>(); T.b2[e] = r.get<uint32_t>(); T.op[e] = r.get<uint32_t>(); T.scale[e] = r.get<double>(); }
        T.herm_left.resize(T.rows); T.phase_left.resize(T.rows);
        T.herm_right.resize(T.cols); T.phase_right.resize(T.cols);
        for (uint32_t i = 0; i < T.rows; ++i) { T.herm_left[i] = r.get<int32_t>(); T.phase_left[i] = r.get<int32_t>(); }
        for (uint32_t i = 0; i < T.cols; ++i) { T.herm_right[i] = r.get<int32_t>(); T.phase_right[i] = r.get<int32_t>(); }
        T.ops = std::make_shared<std::vector<SparseOp>>();
        uint32_t no = r.get<uint32_t>();
        T.ops->resize(no);
        for (auto& o : *T.ops) {
            uint32_t k = r.get<uint32_t>();
            for (uint32_t i = 0; i < k; ++i) { o.in.push_back(r.get<uint32_t>()); o.out.push_back(r.get<uint32_t>()); o.val.push_back(r.get<double>()); }
        }
        T.finalize();
    }
    return m;
}

}  // namespace qcm
