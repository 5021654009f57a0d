// TwoU1 symmetry bookkeeping for the B200 two-site DMRG path (host side).
//
// Charges are (N_up, N_down) pairs (framework/dmrg/block_matrix/symmetry/2u1.h,
// NU1_template<2>).  Ordering is lexicographic (nu1_tpl.h:215-230) and every
// Index is kept sorted in DESCENDING charge order, as the reference's
// indexing_stable.hpp does (index_detail::gt, insert() at destination()).
// ProductBasis offsets follow indexing_stable.hpp:ProductBasis::init: for
// it1 in a, for it2 in b, offset(c1, c2) = running size of the fused sector.
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <utility>
#include <vector>

namespace qcm {

struct Charge {
    int a = 0, b = 0;
    Charge() = default;
    Charge(int x, int y) : a(x), b(y) {}
    Charge operator+(Charge o) const { return {a + o.a, b + o.b}; }
    Charge operator-() const { return {-a, -b}; }
    Charge operator-(Charge o) const { return {a - o.a, b - o.b}; }
    bool operator==(Charge o) const { return a == o.a && b == o.b; }
    bool operator!=(Charge o) const { return !(*this == o); }
    bool operator<(Charge o) const { return a < o.a || (a == o.a && b < o.b); }
    bool operator>(Charge o) const { return o < *this; }
    int particles() const { return a + b; }
};

// Sorted (descending) list of (charge, size) sectors.
struct Index {
    std::vector<std::pair<Charge, std::size_t>> d;

    std::size_t size() const { return d.size(); }
    const std::pair<Charge, std::size_t>& operator[](std::size_t i) const { return d[i]; }
    std::pair<Charge, std::size_t>& operator[](std::size_t i) { return d[i]; }

    // position of charge c, or size() if absent
    std::size_t position(Charge c) const {
        auto it = std::lower_bound(d.begin(), d.end(), c,
                                   [](const std::pair<Charge, std::size_t>& e, Charge x) { return e.first > x; });
        if (it != d.end() && it->first == c) return std::size_t(it - d.begin());
        return d.size();
    }
    bool has(Charge c) const { return position(c) < d.size(); }
    std::size_t size_of(Charge c) const {
        std::size_t p = position(c);
        return p < d.size() ? d[p].second : 0;
    }
    void insert(Charge c, std::size_t s) {
        auto it = std::find_if(d.begin(), d.end(), [&](const std::pair<Charge, std::size_t>& e) { return e.first < c; });
        d.insert(it, {c, s});
    }
    void sort() {
        std::stable_sort(d.begin(), d.end(), [](const std::pair<Charge, std::size_t>& x,
                                                const std::pair<Charge, std::size_t>& y) { return x.first > y.first; });
    }
    std::size_t sum_of_sizes() const {
        std::size_t s = 0;
        for (auto& e : d) s += e.second;
        return s;
    }
    std::vector<std::size_t> sizes() const {
        std::vector<std::size_t> r;
        for (auto& e : d) r.push_back(e.second);
        return r;
    }
    bool operator==(const Index& o) const {
        if (d.size() != o.d.size()) return false;
        for (std::size_t i = 0; i < d.size(); ++i)
            if (d[i].first != o.d[i].first || d[i].second != o.d[i].second) return false;
        return true;
    }
};

// Index product (indexing_stable.hpp operator*): fused charges, sizes multiplied and summed.
inline Index index_product(const Index& i1, const Index& i2) {
    Index r;
    for (auto& x : i1.d)
        for (auto& y : i2.d) {
            Charge c = x.first + y.first;
            std::size_t p = r.position(c);
            if (p < r.size()) r[p].second += x.second * y.second;
            else r.insert(c, x.second * y.second);
        }
    r.sort();
    return r;
}

// adjoin(): negated charges, re-sorted
inline Index adjoin(const Index& in) {
    Index r;
    for (auto& x : in.d) r.insert(-x.first, x.second);
    return r;
}

// Keep only sectors present in both; returns the reduced a (b reduced too).
inline void common_subset(Index& a, Index& b) {
    Index na, nb;
    for (auto& x : a.d) if (b.has(x.first)) na.d.push_back(x);
    for (auto& x : b.d) if (na.has(x.first)) nb.d.push_back(x);
    a = na;
    b = nb;
}

// ProductBasis(a, b, fuse) where fuse(c1, c2) = c1 + c2 (left) or -c1 + c2 (right).
struct ProductBasis {
    std::map<std::pair<std::pair<int, int>, std::pair<int, int>>, std::size_t> off;
    std::map<std::pair<int, int>, std::size_t> tot;
    ProductBasis() = default;
    ProductBasis(const Index& a, const Index& b, bool right = false) {
        for (auto& x : a.d)
            for (auto& y : b.d) {
                Charge pc = right ? (-x.first + y.first) : (x.first + y.first);
                std::size_t& t = tot[{pc.a, pc.b}];
                off[{{x.first.a, x.first.b}, {y.first.a, y.first.b}}] = t;
                t += x.second * y.second;
            }
    }
    std::size_t operator()(Charge c1, Charge c2) const {
        auto it = off.find({{c1.a, c1.b}, {c2.a, c2.b}});
        if (it == off.end()) throw std::runtime_error("ProductBasis: missing charge pair");
        return it->second;
    }
    std::size_t size(Charge pc) const {
        auto it = tot.find({pc.a, pc.b});
        return it == tot.end() ? 0 : it->second;
    }
};

// The QC TwoU1 site basis (models/chem/2u1/model.hpp:49-55): |0>=(0,0), |up>=(1,0),
// |down>=(0,1), |updown>=(1,1), each of multiplicity 1, in descending Index order:
// state 0 = (1,1), 1 = (1,0), 2 = (0,1), 3 = (0,0).
inline Index qc_site_index() {
    Index r;
    r.insert(Charge(0, 0), 1);
    r.insert(Charge(1, 0), 1);
    r.insert(Charge(0, 1), 1);
    r.insert(Charge(1, 1), 1);
    return r;
}

// Flat state numbering of an Index: state = (sector offset) + sub-index.
struct StateMap {
    std::vector<int> sector;   // state -> sector position
    std::vector<int> sub;      // state -> sub-index within sector
    std::vector<int> first;    // sector -> first state
    explicit StateMap(const Index& idx) {
        int s = 0;
        for (std::size_t k = 0; k < idx.size(); ++k) {
            first.push_back(s);
            for (std::size_t j = 0; j < idx[k].second; ++j, ++s) {
                sector.push_back(int(k));
                sub.push_back(int(j));
            }
        }
    }
    int nstates() const { return int(sector.size()); }
};

}  // namespace qcm
