// Jacobi-Davidson eigensolver and the two-site DMRG sweep on the device.
//
// JD (ietl/jacobi.h:386-474, GMRES corrections ietl/gmres.h:78-146, ortho
// vectors ietl_interface_dv.h:94-99): the search space, its H images, the
// GMRES basis and every vector update live in HBM; only the Rayleigh-Ritz
// matrix (<= maxiter^2 numbers), its eigenvector, the GMRES Hessenberg columns
// and a few norms per iteration cross to the host.  Dot products use a fixed-order reduction,
// so a solve is reproducible run to run.
//
// Sweep (optimize/ts_optimize.hpp:114-362): per step, two-site tensor -> H_eff
// plan -> JD -> SVD truncation -> QR/LQ re-gauge -> boundary step, all on one
// stream.  Initialisation: const MPS over allowed_sectors (mps_sectors.h:52-140,
// mps_initializers.h:84-100), MPS::normalize_left (mps.hpp:129-136),
// canonize(0) and the right boundaries (optimize.h:158-195).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "dmrg_dev.hpp"

namespace qcm {

namespace {
double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void download(Ctx& c, const double* d, double* h, std::size_t n) {
    QCM_CUDA(cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    QCM_CUDA(cudaStreamSynchronize(c.s));
}
}  // namespace

namespace {
// GeneratePlaneRotation / ApplyPlaneRotation (ietl/gmres.h:40-66)
void gen_rot(double dx, double dy, double& cs, double& sn) {
    if (dy == 0.0) { cs = 1; sn = 0; }
    else if (std::fabs(dy) > std::fabs(dx)) { const double t = dx / dy; sn = 1.0 / std::sqrt(1.0 + t * t); cs = t * sn; }
    else { const double t = dy / dx; cs = 1.0 / std::sqrt(1.0 + t * t); sn = t * cs; }
}
void apply_rot(double& dx, double& dy, double cs, double sn) {
    const double r0 = cs * dx + sn * dy, r1 = -sn * dx + cs * dy;
    dx = r0;
    dy = r1;
}
}  // namespace

double jacobi_davidson(Ctx& c, HeffPlan& p, double* x, double tol, int maxiter, int& iters, int precision,
                       const JDOptions* opt, int* applies) {
    const bool mixed = precision != 0;
    if (maxiter < 1 || maxiter > 64) throw std::runtime_error("jacobi_davidson: maxiter must be in 1..64");
    const int gm = opt ? opt->gmres : 0;
    if (gm < 0 || gm > JD_MAX_GMRES) throw std::runtime_error("jacobi_davidson: gmres must be in 0..64");
    const uint64_t n = p.x_len, ld = (n + 31) / 32 * 32;
    // at most n - 1 ortho vectors (solver/ietl_jacobi_davidson.h:41-42)
    int no = opt ? opt->n_ortho : 0;
    if (no < 0) throw std::runtime_error("jacobi_davidson: negative ortho vector count");
    if (uint64_t(no) >= n) no = n ? int(n - 1) : 0;
    if (no > 0 && (!opt->ortho || opt->ortho_ld < n)) throw std::runtime_error("jacobi_davidson: bad ortho vectors");
    // V[0..maxiter), VA[0..maxiter), u, r, the ortho vectors, the GMRES basis (gm + 1) and the
    // correction operator's temporary
    // (+ three vectors for the mixed form's FP64 correction: H u, t, H t)
    const uint64_t nmx = mixed ? 3 : 0;
    const uint64_t nvec = 2 * uint64_t(maxiter) + 2 + uint64_t(no) + (gm > 0 ? uint64_t(gm) + 2 : 0) + nmx;
    Ctx::ensure(c.jd, nvec * ld);
    Ctx::ensure(c.scal, 256 + 64 * uint64_t(DOT_PARTS));
    Ctx::ensure(c.coef, 64);
    double* V = c.jd.get();
    double* VA = V + uint64_t(maxiter) * ld;
    double* u = VA + uint64_t(maxiter) * ld;
    double* r = u + ld;
    double* O = r + ld;
    double* G = O + uint64_t(no) * ld;
    double* tmp = G + uint64_t(gm + 1) * ld;
    double* MX = V + (nvec - nmx) * ld;
    // scalar slots: 0-1 norms, 2.. MGS dots, 80.. Rayleigh-Ritz column, 160-164 residual / Rayleigh
    // quotient, 170.. GMRES Hessenberg column and |w|^2, 241-242 operator dots, 243-246 projections
    double* sc = c.scal.get();
    double* dsc = sc + 256;  // dot-product partials
    auto Vi = [&](int i) { return V + uint64_t(i) * ld; };
    auto VAi = [&](int i) { return VA + uint64_t(i) * ld; };
    auto Oi = [&](int i) { return O + uint64_t(i) * ld; };
    auto Gi = [&](int i) { return G + uint64_t(i) * ld; };
    int napply = 0;
    auto apply = [&](const double* in, double* out) {
        if (mixed) heff_apply_device_mixed(p, in, out, nullptr, precision == 2);
        else heff_apply_device(p, in, out);
        ++napply;
    };
    // ortho vectors: copies, Gram-Schmidt among themselves in order (ietl_jacobi_davidson.h:43-47)
    std::vector<double> inv_oo(std::size_t(no > 0 ? no : 0));
    for (int a = 0; a < no; ++a) {
        QCM_CUDA(cudaMemcpyAsync(Oi(a), opt->ortho + uint64_t(a) * opt->ortho_ld, n * sizeof(double),
                                 cudaMemcpyDeviceToDevice, c.s));
        for (int b = 0; b < a; ++b) {
            dev_dots(Oi(b), 0, 1, Oi(a), n, sc + 243, dsc, c.s);
            dev_axpy_dscalar(sc + 243, -inv_oo[b], Oi(b), Oi(a), n, c.s);
        }
        dev_dots(Oi(a), 0, 1, Oi(a), n, sc + 244, dsc, c.s);
        double oo = 0.0;
        download(c, sc + 244, &oo, 1);
        if (!(oo > 0.0) || !std::isfinite(oo))
            throw std::runtime_error("jacobi_davidson: ortho vector of zero norm after Gram-Schmidt");
        inv_oo[a] = 1.0 / oo;
    }
    // t -= (o.t)/(o.o) o for each ortho vector in turn
    auto project = [&](double* t) {
        for (int a = 0; a < no; ++a) {
            dev_dots(Oi(a), 0, 1, t, n, sc + 243, dsc, c.s);
            dev_axpy_dscalar(sc + 243, -inv_oo[a], Oi(a), t, n, c.s);
        }
    };
    // The mixed form's FP64 residual correction (the precision form): u (the mixed solve's vector) gets an
    // FP64 apply for its Rayleigh quotient and residual; then, while that residual is above tol |theta|
    // and steps remain, one Jacobi-Davidson step in FP64: t = -r + (r.u)/(u.u) u projected and made
    // orthogonal to u, Rayleigh-Ritz on span{u, t} (2 x 2, FP64 H.psi of t).  Returns the FP64
    // eigenvalue, u normalised.
    const double mixed_floor = opt ? opt->mixed_floor : 0.0;
    const int mixed_refine = opt ? opt->mixed_refine : 0;
    int fp64_applies = 0;
    double rn_prev = std::numeric_limits<double>::infinity();
    auto fp64_correction = [&](double* uu, double* rr, double th) -> double {
        double* Hu = MX;
        double* t = MX + ld;
        double* Ht = MX + 2 * ld;
        dev_dots(uu, 0, 1, uu, n, sc + 164, dsc, c.s);
        double q[3];
        download(c, sc + 164, q, 1);
        dev_axpby(1.0 / std::sqrt(q[0]), uu, 0.0, uu, n, c.s);
        heff_apply_device(p, uu, Hu);
        ++fp64_applies;
        project(Hu);
        dev_dots(uu, 0, 1, Hu, n, sc + 163, dsc, c.s);
        download(c, sc + 163, q, 1);
        th = q[0];
        for (int k = 0;; ++k) {
            // r = Hu - theta u (FP64)
            QCM_CUDA(cudaMemcpyAsync(rr, Hu, n * sizeof(double), cudaMemcpyDeviceToDevice, c.s));
            dev_axpby(-th, uu, 1.0, rr, n, c.s);
            dev_dots(rr, 0, 1, rr, n, sc + 160, dsc, c.s);
            dev_dots(rr, 0, 1, uu, n, sc + 161, dsc, c.s);
            download(c, sc + 160, q, 2);
            const double rn64 = std::sqrt(q[0]);
            if (k >= mixed_refine || rn64 <= tol * std::fabs(th) || rn64 < tol) break;
            // t = -r + (r.u) u, projected, orthogonal to u, normalised
            dev_axpby(-1.0, rr, 0.0, t, n, c.s);
            dev_axpby(q[1], uu, 1.0, t, n, c.s);
            project(t);
            dev_dots(uu, 0, 1, t, n, sc + 165, dsc, c.s);
            dev_axpy_dscalar(sc + 165, -1.0, uu, t, n, c.s);
            dev_dots(t, 0, 1, t, n, sc + 166, dsc, c.s);
            download(c, sc + 166, q, 1);
            if (!(q[0] > 0.0)) break;
            dev_axpby(1.0 / std::sqrt(q[0]), t, 0.0, t, n, c.s);
            heff_apply_device(p, t, Ht);
            ++fp64_applies;
            project(Ht);
            dev_dots(t, 0, 1, Ht, n, sc + 167, dsc, c.s);
            dev_dots(uu, 0, 1, Ht, n, sc + 168, dsc, c.s);
            download(c, sc + 167, q, 2);
            // lowest eigenpair of [[th, b], [b, d]]
            const double a11 = th, b = q[1], d = q[0];
            const double mid = 0.5 * (a11 + d), half = 0.5 * (a11 - d);
            const double lam = mid - std::sqrt(half * half + b * b);
            // eigenvector (cu, ct) of lam, normalised
            double cu = b, ct = lam - a11;
            if (std::fabs(cu) + std::fabs(ct) == 0.0) { cu = 1.0; ct = 0.0; }
            const double nrm = std::sqrt(cu * cu + ct * ct);
            cu /= nrm;
            ct /= nrm;
            dev_axpby(ct, t, cu, uu, n, c.s);
            dev_axpby(ct, Ht, cu, Hu, n, c.s);
            th = lam;
        }
        return th;
    };
    QCM_CUDA(cudaMemcpyAsync(Vi(0), x, n * sizeof(double), cudaMemcpyDeviceToDevice, c.s));
    project(Vi(0));
    std::vector<double> M(std::size_t(maxiter) * maxiter, 0.0), s;
    int it = 0;
    double theta = 0.0;
    // (I - uu*)(A - theta)(I - uu*) x -> y (jcd_solver_operator, ietl/jacobi.h:249-268; u has unit norm)
    auto op = [&](const double* xin, double* y) {
        dev_dots(u, 0, 1, xin, n, sc + 241, dsc, c.s);
        QCM_CUDA(cudaMemcpyAsync(tmp, xin, n * sizeof(double), cudaMemcpyDeviceToDevice, c.s));
        dev_axpy_dscalar(sc + 241, -1.0, u, tmp, n, c.s);
        apply(tmp, y);
        dev_axpby(-theta, tmp, 1.0, y, n, c.s);
        dev_dots(u, 0, 1, y, n, sc + 242, dsc, c.s);
        dev_axpy_dscalar(sc + 242, -1.0, u, y, n, c.s);
    };
    // ietl_gmres::operator() (ietl/gmres.h:92-146) for b = -r from xt (in: t0, out: the solution).
    // A break at inner step i keeps the first i directions (Update(H, s, i)), as the reference does.
    auto gmres = [&](double* xt, double abs_tol) {
        const int m = gm;
        std::vector<double> sv(std::size_t(m) + 1, 0.0), cs(std::size_t(m) + 1, 0.0), sn(std::size_t(m) + 1, 0.0);
        std::vector<double> H(std::size_t(m + 1) * (m + 1), 0.0);
        auto h = [&](int i, int j) -> double& { return H[std::size_t(i) + std::size_t(j) * (m + 1)]; };
        op(xt, Gi(0));
        dev_axpby(-1.0, r, -1.0, Gi(0), n, c.s);  // b - A x0
        dev_dots(Gi(0), 0, 1, Gi(0), n, sc + 246, dsc, c.s);
        double s0 = 0.0;
        download(c, sc + 246, &s0, 1);
        sv[0] = std::sqrt(s0);
        if (std::fabs(sv[0]) < abs_tol) return;
        dev_axpby(1.0 / sv[0], Gi(0), 0.0, Gi(0), n, c.s);
        int i = 0;
        std::vector<double> col(std::size_t(m) + 1);
        for (; i + 1 < m; ++i) {
            double* w = Gi(i + 1);
            op(Gi(i), w);
            for (int k = 0; k <= i; ++k) {
                dev_dots(Gi(k), 0, 1, w, n, sc + 170 + k, dsc, c.s);
                dev_axpy_dscalar(sc + 170 + k, -1.0, Gi(k), w, n, c.s);
            }
            dev_dots(w, 0, 1, w, n, sc + 170 + i + 1, dsc, c.s);
            download(c, sc + 170, col.data(), std::size_t(i) + 2);
            for (int k = 0; k <= i; ++k) h(k, i) = col[k];
            h(i + 1, i) = std::sqrt(col[i + 1]);
            // an exact breakdown leaves w = 0: the rotation below zeroes the residual and ends the loop
            // before the direction would be used
            if (h(i + 1, i) != 0.0) dev_axpby(1.0 / h(i + 1, i), w, 0.0, w, n, c.s);
            for (int k = 0; k < i; ++k) apply_rot(h(k, i), h(k + 1, i), cs[k], sn[k]);
            gen_rot(h(i, i), h(i + 1, i), cs[i], sn[i]);
            apply_rot(h(i, i), h(i + 1, i), cs[i], sn[i]);
            apply_rot(sv[i], sv[i + 1], cs[i], sn[i]);
            if (std::fabs(sv[i + 1]) < abs_tol) break;
        }
        if (i == 0) return;
        std::vector<double> y(sv.begin(), sv.begin() + i);
        for (int a = i - 1; a >= 0; --a) {
            y[a] /= h(a, a);
            for (int b = a - 1; b >= 0; --b) y[b] -= h(b, a) * y[a];
        }
        QCM_CUDA(cudaMemcpyAsync(c.coef.get(), y.data(), y.size() * sizeof(double), cudaMemcpyHostToDevice, c.s));
        dev_lincomb(G, ld, uint32_t(i), c.coef.get(), n, xt, true, c.s);
    };
    while (true) {
        double* t = Vi(it);
        // modified Gram-Schmidt against V[0..it), repeated once if the norm dropped below 1/4
        auto mgs = [&]() {
            for (int i = 0; i < it; ++i) {
                dev_dots(Vi(i), 0, 1, t, n, sc + 2 + i, dsc, c.s);
                dev_axpy_dscalar(sc + 2 + i, -1.0, Vi(i), t, n, c.s);
            }
            dev_dots(t, 0, 1, t, n, sc + 1, dsc, c.s);
        };
        dev_dots(t, 0, 1, t, n, sc, dsc, c.s);
        mgs();
        double h2[2];
        download(c, sc, h2, 2);
        double tau = std::sqrt(h2[0]), tn = std::sqrt(h2[1]);
        if (tn < 0.25 * tau) {
            mgs();
            download(c, sc + 1, h2, 1);
            tn = std::sqrt(h2[0]);
        }
        if (no > 0) {
            project(t);
            dev_dots(t, 0, 1, t, n, sc + 245, dsc, c.s);
            download(c, sc + 245, h2, 1);
            tn = std::sqrt(h2[0]);
        }
        dev_axpby(1.0 / tn, t, 0.0, t, n, c.s);
        apply(t, VAi(it));
        // column it of the projected matrix: <V_i, A V_it>
        dev_dots(V, ld, uint32_t(it + 1), VAi(it), n, sc + 80, dsc, c.s);
        std::vector<double> col(it + 1);
        download(c, sc + 80, col.data(), col.size());
        for (int i = 0; i <= it; ++i) M[i + std::size_t(it) * maxiter] = col[i];
        sym_lowest_eigenpair(M.data(), maxiter, it + 1, theta, s);
        QCM_CUDA(cudaMemcpyAsync(c.coef.get(), s.data(), s.size() * sizeof(double), cudaMemcpyHostToDevice, c.s));
        dev_lincomb(V, ld, uint32_t(it + 1), c.coef.get(), n, u, false, c.s);
        // r = A u - theta u, A u projected against the ortho vectors
        dev_lincomb(VA, ld, uint32_t(it + 1), c.coef.get(), n, r, false, c.s);
        project(r);
        dev_axpby(-theta, u, 1.0, r, n, c.s);
        dev_dots(r, 0, 1, r, n, sc + 160, dsc, c.s);
        dev_dots(r, 0, 1, u, n, sc + 161, dsc, c.s);
        dev_dots(u, 0, 1, u, n, sc + 162, dsc, c.s);
        double h3[3];
        download(c, sc + 160, h3, 3);
        ++it;
        const double rn = std::sqrt(h3[0]);
        // The mixed iterations follow the FP64 stopping rule, so that a sweep in the mixed form takes
        // the FP64 sweep's path; with a floor (mixed_floor > 0) they also stop once the residual is
        // below mixed_floor |theta| and no longer halves: below the mixed H.psi's relative error
        // (~1e-7) the residual is noise, and a converged step then costs fewer applies
        const bool stalled = mixed && mixed_floor > 0.0 && rn <= mixed_floor * std::fabs(theta) && rn > 0.5 * rn_prev;
        rn_prev = rn;
        if (rn <= tol * std::fabs(theta) || rn < tol || it >= maxiter || stalled) {
            if (mixed) {
                check_mixed(p);
                theta = fp64_correction(u, r, theta);
            }
            QCM_CUDA(cudaMemcpyAsync(x, u, n * sizeof(double), cudaMemcpyDeviceToDevice, c.s));
            iters = it;
            if (applies) *applies = napply;
            if (opt) const_cast<JDOptions*>(opt)->fp64_applies = fp64_applies;
            return theta;
        }
        // correction t0 = -r + (r.u)/(u.u) u, then GMRES on -r with abs_tol 2^-(it+1)
        dev_axpby(-1.0, r, 0.0, Vi(it), n, c.s);
        dev_axpby(h3[1] / h3[2], u, 1.0, Vi(it), n, c.s);
        if (gm > 0) gmres(Vi(it), 1.0 / std::pow(2.0, double(it + 1)));
    }
}

// ---------------------------------------------------------------------------
std::unique_ptr<DevBoundary> trivial_boundary(const Index& idx, uint32_t aux_dim, cudaStream_t s) {
    auto B = std::make_unique<DevBoundary>();
    BoundaryIndexH& x = B->idx;
    x.bra = idx; x.ket = idx; x.aux = aux_dim;
    for (uint32_t i = 0; i < idx.size(); ++i) {
        const uint32_t ls = uint32_t(idx[i].second);
        x.cbra.push_back(i); x.cket.push_back(i); x.lsz.push_back(ls); x.rsz.push_back(ls);
        x.nb.push_back(aux_dim); x.tr.push_back(0);
        for (uint32_t b = 0; b < aux_dim; ++b) { x.offsets.push_back(int64_t(b) * ls * ls); x.cscale.push_back(1.0); }
    }
    x.finish();
    B->data.alloc(x.total ? x.total : 1);
    dev_fill(B->data.get(), x.total ? x.total : 1, 1.0, s);
    return B;
}

namespace {
// allowed_sectors (mps_sectors.h:52-140)
std::vector<Index> allowed_sectors(int L, const Index& phys, Charge right_end, std::size_t Mmax) {
    Index physc = phys;
    physc.sort();
    Charge maxc = physc.d.front().first, minc = physc.d.back().first;
    if (minc > maxc) std::swap(maxc, minc);
    Charge maxt, mint;
    for (int i = 0; i < L; ++i) { maxt = maxt + maxc; mint = mint + minc; }
    std::vector<Index> la(L + 1), ra(L + 1), allowed(L + 1);
    la[0].d.push_back({Charge(0, 0), 1});
    ra[L].d.push_back({right_end, 1});
    Charge cmaxi = maxt, cmini = mint;
    for (int i = 1; i <= L; ++i) {
        la[i] = index_product(phys, la[i - 1]);
        cmaxi = cmaxi - maxc;
        cmini = cmini - minc;
        Index keep;
        for (auto& e : la[i].d) {
            if ((e.first + cmaxi) < right_end) continue;
            if ((e.first + cmini) > right_end) continue;
            keep.d.push_back({e.first, std::min(Mmax, e.second)});
        }
        la[i] = keep;
    }
    cmaxi = maxt; cmini = mint;
    for (int i = L - 1; i >= 0; --i) {
        ra[i] = index_product(adjoin(phys), ra[i + 1]);
        cmaxi = cmaxi - maxc;
        cmini = cmini - minc;
        Index keep;
        for (auto& e : ra[i].d) {
            if ((e.first - cmaxi) > Charge(0, 0)) continue;
            if ((e.first - cmini) < Charge(0, 0)) continue;
            keep.d.push_back({e.first, std::min(Mmax, e.second)});
        }
        ra[i] = keep;
    }
    for (int i = 0; i <= L; ++i) {
        Index a = la[i], b = ra[i];
        common_subset(a, b);
        for (auto& e : a.d) e.second = std::min(Mmax, std::min(la[i].size_of(e.first), ra[i].size_of(e.first)));
        allowed[i] = a;
    }
    return allowed;
}

// MPSTensor(sd, ld, rd, fillrand = false, val) (mpstensor.hpp:40-71), left-paired blocks of `val`
DMPS const_tensor(Ctx& c, const Index& sd, const Index& ld, const Index& rd, double val) {
    DMPS t;
    t.phys = sd;
    Index lb = index_product(sd, ld), rb = rd;
    common_subset(lb, rb);
    t.right = rb;
    Index possible = index_product(adjoin(sd), t.right), ltemp = ld;
    common_subset(ltemp, possible);
    t.left = ltemp;
    lb.sort(); rb.sort(); t.left.sort(); t.right.sort();
    t.right_paired = false;
    t.b = layout_left_paired(t.phys, t.left, t.right);
    for (std::size_t k = 0; k < t.b.n(); ++k)
        if (t.b.rows[k] != lb.size_of(t.b.rc[k])) throw std::runtime_error("const MPS: left basis reduced by the right basis");
    t.b.allocate(c.s, true);
    for (std::size_t k = 0; k < t.b.n(); ++k) dev_fill(t.b.d.get() + t.b.off[k], t.b.elems(k), val, c.s);
    return t;
}
// a right-paired site tensor in the packed block layout of the H_eff vector
DMPS packed_right(Ctx& c, const DMPS& t) {
    if (!t.right_paired) throw std::runtime_error("DMRG: expected a right-paired site tensor");
    DMPS o;
    o.phys = t.phys; o.left = t.left; o.right = t.right; o.right_paired = true;
    o.b = layout_right_paired(t.phys, t.left, t.right, true);
    o.b.allocate(c.s, true);
    std::vector<CopyJob> cj;
    for (std::size_t k = 0; k < o.b.n(); ++k) {
        const std::size_t ks = t.b.find_l(o.b.lc[k]);
        if (ks == t.b.n()) continue;
        if (t.b.rows[ks] != o.b.rows[k] || t.b.cols[ks] != o.b.cols[k])
            throw std::runtime_error("DMRG: site tensor block differs from its right-paired layout");
        cj.push_back(CopyJob{t.b.off[ks], o.b.off[k], o.b.rows[k], o.b.cols[k], t.b.rows[ks], o.b.rows[k], 0, 0});
    }
    if (cj.size() != t.b.n()) throw std::runtime_error("DMRG: site tensor has blocks outside its indices");
    if (!cj.empty()) batched_copy(cj, t.b.d.get(), t.b.total, o.b.d.get(), o.b.total, c.cjobs, c.s);
    return o;
}
}  // namespace

DevDMRG::DevDMRG(const std::vector<MPOTensor>& single, const std::vector<MPOTensor>& twosite, int nup, int ndown,
                 const DMRGParams& prm, cudaStream_t s)
    : mpo(single), ts_mpo(twosite), p(prm) {
    c.s = s;
    QCM_CUDA(cudaGetDevice(&c.device));
    L = int(mpo.size());
    if (L < 2 || int(ts_mpo.size()) != L - 1) throw std::runtime_error("DMRG: need L >= 2 site tensors and L - 1 two-site tensors");
    const Index& phys = mpo[0].phys;
    std::vector<Index> allowed = allowed_sectors(L, phys, Charge(nup, ndown), p.init_bond_dimension);
    mps.resize(L);
    for (int i = 0; i < L; ++i) {
        mps[i] = const_tensor(c, phys, allowed[i], allowed[i + 1], 1.0);
        scale(c, mps[i].b, 1.0 / std::sqrt(norm2(c, mps[i].b)));
    }
    for (int i = 0; i < L - 1; ++i) {
        DBlocks t = normalize_left(c, mps[i]);
        multiply_from_left(c, mps[i + 1], t);
        scale(c, mps[i + 1].b, 1.0 / std::sqrt(norm2(c, mps[i + 1].b)));
    }
    normalize_left(c, mps[L - 1]);
    for (int i = L - 1; i > 0; --i) {
        DBlocks t = normalize_right(c, mps[i]);
        multiply_from_right(c, mps[i - 1], t);
        scale(c, mps[i - 1].b, 1.0 / std::sqrt(norm2(c, mps[i - 1].b)));
    }
    init_boundaries();
}

DevDMRG::DevDMRG(const std::vector<MPOTensor>& single, const std::vector<MPOTensor>& twosite, std::vector<DMPS> sites,
                 const DMRGParams& prm, cudaStream_t s, int initial_site)
    : mpo(single), ts_mpo(twosite), mps(std::move(sites)), p(prm) {
    c.s = s;
    QCM_CUDA(cudaGetDevice(&c.device));
    L = int(mpo.size());
    if (L < 2 || int(ts_mpo.size()) != L - 1 || int(mps.size()) != L)
        throw std::runtime_error("DMRG: need L site tensors, L MPO tensors and L - 1 two-site tensors");
    for (int i = 0; i + 1 < L; ++i)
        if (!(mps[i].right == mps[i + 1].left)) throw std::runtime_error("DMRG: site tensors do not share their bond indices");
    const int last = p.single_site ? L - 1 : L - 2;
    if (initial_site < 0 || initial_site > last) throw std::runtime_error("DMRG: initial site outside the left-to-right half-sweep");
    init_boundaries(initial_site);
}

void DevDMRG::init_boundaries(int site) {
    left_.resize(L + 1);
    right_.resize(L + 1);
    left_[0] = trivial_boundary(mps[0].left, mpo[0].rows, c.s);
    right_[L] = trivial_boundary(mps[L - 1].right, mpo[L - 1].cols, c.s);
    for (int i = 0; i < site; ++i) {
        make_left_paired(c, mps[i]);
        DMPS ket = right_paired_copy(c, mps[i]);
        left_[i + 1] = boundary_step_left(c, *left_[i], ket, mps[i], mpo[i], true);
    }
    for (int i = L - 1; i >= site; --i) {
        make_right_paired(c, mps[i]);
        right_[i] = boundary_step_right(c, *right_[i + 1], mps[i], mpo[i], true);
    }
    next_step = site;
    QCM_CUDA(cudaStreamSynchronize(c.s));
    bnd_trim(site);
}

void DevDMRG::set_ortho(std::vector<std::vector<DMPS>> states_rp) {
    if (next_step != 0) throw std::runtime_error("DMRG: ortho states are set at the start of a sweep");
    for (auto& st : states_rp) {
        if (int(st.size()) != L) throw std::runtime_error("DMRG: an ortho state has the wrong length");
        for (int i = 0; i < L; ++i)
            if (!st[i].right_paired || !(st[i].phys == mps[i].phys)) throw std::runtime_error("DMRG: ortho state site tensor mismatch");
        if (!(st[0].left == mps[0].left) || !(st[L - 1].right == mps[L - 1].right))
            throw std::runtime_error("DMRG: ortho state with different end sectors");
    }
    ortho_rp = std::move(states_rp);
    const std::size_t n = ortho_rp.size();
    ortho_lp.clear();
    ortho_lp.resize(n);
    ortho_left_.clear();
    ortho_left_.resize(n);
    ortho_right_.clear();
    ortho_right_.resize(n);
    for (std::size_t o = 0; o < n; ++o) {
        for (int i = 0; i < L; ++i) ortho_lp[o].push_back(left_paired_copy(c, ortho_rp[o][i]));
        ortho_left_[o].resize(L + 1);
        ortho_right_[o].resize(L + 1);
        ortho_left_[o][0] = unit_blocks(c, mps[0].left);
        ortho_right_[o][L] = unit_blocks(c, mps[L - 1].right);
        for (int i = L - 1; i >= 0; --i) {
            make_right_paired(c, mps[i]);
            ortho_right_[o][i] = ortho_right_step(c, mps[i], ortho_lp[o][i], ortho_right_[o][i + 1]);
        }
    }
    QCM_CUDA(cudaStreamSynchronize(c.s));
}

double DevDMRG::expectation(const std::vector<MPOTensor>& W) {
    if (next_step != 0) throw std::runtime_error("DMRG: expectation values are taken between sweeps");
    if (int(W.size()) != L) throw std::runtime_error("DMRG: operator MPO of the wrong length");
    std::unique_ptr<DevBoundary> B = trivial_boundary(mps[0].left, W[0].rows, c.s);
    for (int k = 0; k < L; ++k) {
        if (!(W[k].phys == mps[k].phys)) throw std::runtime_error("DMRG: operator MPO with another physical basis");
        make_left_paired(c, mps[k]);
        DMPS ket = right_paired_copy(c, mps[k]);
        B = boundary_step_left(c, *B, ket, mps[k], W[k], true);
    }
    // the last boundary: one cohort (the end sector, dimension 1) with W[L-1].cols = 1 block of 1 x 1
    const BoundaryIndexH& x = B->idx;
    if (x.n_cohorts() != 1 || x.aux != 1 || x.lsz[0] != 1 || x.rsz[0] != 1 || x.offsets[0] < 0)
        throw std::runtime_error("DMRG: unexpected final boundary of an expectation value");
    const uint64_t at = x.data_off[0] + uint64_t(x.offsets[0]);
    if (at >= B->data.size()) throw std::runtime_error("DMRG: final boundary outside its buffer");
    double v = 0.0;
    QCM_CUDA(cudaMemcpyAsync(&v, B->data.get() + at, sizeof(double), cudaMemcpyDeviceToHost, c.s));
    QCM_CUDA(cudaStreamSynchronize(c.s));
    // sites 1 .. L-1 are right-normalised between sweeps: the norm lives in site 0
    const double n2 = norm2(c, mps[0].b);
    if (!(n2 > 0.0)) throw std::runtime_error("DMRG: zero state");
    return v / n2;
}

std::vector<std::vector<double>> DevDMRG::mpo_gradient(const std::vector<MPOTensor>& W) {
    if (next_step != 0) throw std::runtime_error("DMRG: gradients are taken between sweeps");
    if (int(W.size()) != L) throw std::runtime_error("DMRG: gradient MPO of the wrong length");
    for (int k = 0; k < L; ++k)
        if (!(W[k].phys == mps[k].phys)) throw std::runtime_error("DMRG: gradient MPO with another physical basis");
    // E = <Psi|W|Psi> / <Psi|Psi> is linear in each site tensor of W, so dE/d scale_e for an entry of
    // site k is the single-site H_eff of site k differentiated in that scale, x . (dH_eff/ds_e) x / x.x,
    // with x the orthogonality centre at site k (the other sites orthonormal).  The centre moves
    // through a copy of the MPS (right-normalised on sites 1 .. L-1 between sweeps): QR of site k,
    // R into site k + 1, one left boundary step of W; the right boundaries of W are built first.
    std::vector<DMPS> m;
    m.reserve(std::size_t(L));
    for (int k = 0; k < L; ++k) {
        make_right_paired(c, mps[k]);
        m.push_back(right_paired_copy(c, mps[k]));
    }
    std::vector<std::unique_ptr<DevBoundary>> R(std::size_t(L) + 1);
    R[std::size_t(L)] = trivial_boundary(m[std::size_t(L) - 1].right, W[std::size_t(L) - 1].cols, c.s);
    for (int k = L - 1; k >= 1; --k) R[std::size_t(k)] = boundary_step_right(c, *R[std::size_t(k) + 1], m[std::size_t(k)], W[std::size_t(k)], true);
    std::unique_ptr<DevBoundary> Lb = trivial_boundary(m[0].left, W[0].rows, c.s);
    std::vector<std::vector<double>> grad(static_cast<std::size_t>(L));
    for (int k = 0; k < L; ++k) {
        DMPS& a = m[std::size_t(k)];
        make_right_paired(c, a);
        DMPS x = packed_right(c, a);
        {
            auto plan = build_heff_plan(*Lb, *R[std::size_t(k) + 1], W[std::size_t(k)], x.phys, x.left, x.right, false);
            plan->stream = c.s;
            if (plan->x_len != x.b.total) throw std::runtime_error("DMRG: site tensor layout differs from the gradient plan");
            const uint64_t nt = heff_adjoint_terms(*plan);
            if (nt != W[std::size_t(k)].b1.size()) throw std::runtime_error("DMRG: gradient plan without every MPO entry");
            upload_plan(*plan);
            const double n2 = norm2(c, x.b);
            if (!(n2 > 0.0)) throw std::runtime_error("DMRG: zero state");
            DBuf<double> cb(nt + 1);
            heff_adjoint_device(*plan, x.b.d.get(), x.b.d.get(), nullptr, cb.get());
            std::vector<double>& g = grad[std::size_t(k)];
            g.resize(nt);
            if (nt) QCM_CUDA(cudaMemcpyAsync(g.data(), cb.get(), nt * sizeof(double), cudaMemcpyDeviceToHost, c.s));
            QCM_CUDA(cudaStreamSynchronize(c.s));
            for (double& v : g) v /= n2;
        }
        R[std::size_t(k) + 1].reset();
        if (k + 1 < L) {
            DBlocks Rm = normalize_left(c, a);
            multiply_from_left(c, m[std::size_t(k) + 1], Rm);
            make_left_paired(c, a);
            DMPS ket = right_paired_copy(c, a);
            Lb = boundary_step_left(c, *Lb, ket, a, W[std::size_t(k)], true);
        }
    }
    QCM_CUDA(cudaStreamSynchronize(c.s));
    return grad;
}

BStepCache* DevDMRG::bstep_cache_for(int step) {
    if (bstep_cache_.size() != std::size_t(steps_per_sweep())) {
        bstep_cache_.clear();
        bstep_cache_.resize(std::size_t(steps_per_sweep()));
        bstep_cache_bytes_ = 0;
    }
    if (!bstep_cache_budget_) {
        size_t free_b = 0, total_b = 0;
        QCM_CUDA(cudaMemGetInfo(&free_b, &total_b));
        bstep_cache_budget_ = uint64_t(total_b) / 16;
    }
    BStepCache& e = bstep_cache_[std::size_t(step)];
    bstep_cache_bytes_ -= e.bytes;
    return &e;
}

void DevDMRG::bnd_use(DevBoundary* b) {
    if (!b || b->data.get() || !b->host) return;
    b->data.alloc(b->host_len);
    QCM_CUDA(cudaMemcpyAsync(b->data.get(), b->host.get(), b->host_len * sizeof(double), cudaMemcpyHostToDevice, c.s));
    ++st.boundaries_fetched;
}

void DevDMRG::bnd_trim(int next) {
    const int n = steps_per_sweep();
    next = ((next % n) + n) % n;
    int lb = 0, rb = 0;  // the boundaries the next step reads
    if (p.single_site) {
        const int site = next < L ? next : 2 * L - 1 - next;
        lb = site; rb = site + 1;
    } else {
        int lr = 0, s1 = 0, s2 = 0;
        step_sites(next, lr, s1, s2);
        lb = s1; rb = s2 + 1;
    }
    auto bytes = [](const DevBoundary* b) { return b && b->data.get() ? uint64_t(b->data.size()) * sizeof(double) : 0; };
    uint64_t tot = 0;
    for (const auto& b : left_) tot += bytes(b.get());
    for (const auto& b : right_) tot += bytes(b.get());
    while (boundary_budget && tot > boundary_budget) {
        // the device-resident boundary farthest from the next step's two
        DevBoundary* far = nullptr;
        int fd = -1;
        for (int i = 0; i < int(left_.size()); ++i)
            if (i != lb && bytes(left_[std::size_t(i)].get()) && std::abs(i - lb) > fd) { fd = std::abs(i - lb); far = left_[std::size_t(i)].get(); }
        for (int j = 0; j < int(right_.size()); ++j)
            if (j != rb && bytes(right_[std::size_t(j)].get()) && std::abs(j - rb) > fd) { fd = std::abs(j - rb); far = right_[std::size_t(j)].get(); }
        if (!far) break;
        tot -= bytes(far);
        if (!far->host) {
            double* h = nullptr;
            const uint64_t len = far->data.size();
            QCM_CUDA(cudaMallocHost(&h, len * sizeof(double)));
            far->host = std::shared_ptr<double>(h, [](double* q) { cudaFreeHost(q); });
            far->host_len = len;
            QCM_CUDA(cudaMemcpyAsync(h, far->data.get(), len * sizeof(double), cudaMemcpyDeviceToHost, c.s));
            QCM_CUDA(cudaStreamSynchronize(c.s));
        }
        far->data.reset();
        ++st.boundaries_offloaded;
    }
    st.boundary_bytes_peak = std::max(st.boundary_bytes_peak, tot);
}

void DevDMRG::bstep_cache_done(int step) {
    BStepCache& e = bstep_cache_[std::size_t(step)];
    ++(e.hit ? st.bsteps_reused : st.bsteps_built);
    if (bstep_cache_bytes_ + e.bytes > bstep_cache_budget_) {
        e.plan.reset();
        e.key = 0;
        e.bytes = 0;
    }
    bstep_cache_bytes_ += e.bytes;
}

std::unique_ptr<HeffPlan> DevDMRG::plan_for(int step, const DevBoundary& Lb, const DevBoundary& Rb, const MPOTensor& W,
                                            const Index& phys, const Index& left, const Index& right, uint64_t& key,
                                            bool& resident) {
    key = plan_structure_key(Lb, Rb, phys, left, right);
    if (plan_cache_.size() != std::size_t(steps_per_sweep())) plan_cache_.resize(std::size_t(steps_per_sweep()));
    CachedPlan& e = plan_cache_[std::size_t(step)];
    resident = false;
    if (e.plan && e.key == key) {
        std::unique_ptr<HeffPlan> p = std::move(e.plan);
        rebind_plan(*p, Lb, Rb);
        resident = e.resident > 0;
        plan_cache_bytes_ -= e.resident;
        e.resident = 0;
        ++st.plans_reused;
        return p;
    }
    e.plan.reset();
    plan_cache_bytes_ -= e.resident;
    e.resident = 0;
    ++st.plans_built;
    return build_heff_plan(Lb, Rb, W, phys, left, right, false);
}

void DevDMRG::keep_plan(int step, std::unique_ptr<HeffPlan> plan, uint64_t key) {
    if (!plan_cache_budget_) {
        // a quarter of the device's memory for the work lists and coefficient blocks kept between sweeps
        size_t free_b = 0, total_b = 0;
        QCM_CUDA(cudaMemGetInfo(&free_b, &total_b));
        plan_cache_budget_ = uint64_t(total_b) / 4;
    }
    CachedPlan& e = plan_cache_[std::size_t(step)];
    const uint64_t rb = plan_resident_bytes(*plan);
    if (plan_cache_bytes_ + rb <= plan_cache_budget_) {
        release_plan_scratch(*plan);
        e.resident = rb;
        plan_cache_bytes_ += rb;
    } else {
        release_plan_device(*plan);
        e.resident = 0;
    }
    plan->L = nullptr;
    plan->R = nullptr;
    plan->cg.b_cs = nullptr;
    e.plan = std::move(plan);
    e.key = key;
}

void DevDMRG::step_sites(int _site, int& lr, int& site1, int& site2) const {
    const int site = (_site < L - 1) ? _site : 2 * L - 2 - _site;
    if (_site < L - 1) { lr = 1; site1 = site; site2 = site + 1; }
    else { lr = -1; site1 = site - 1; site2 = site; }
}

double DevDMRG::solve(HeffPlan& plan, DMPS& x, const std::function<void(std::size_t, double*)>& make_ortho) {
    const double t1 = now_s();
    int iters = 0, napply = 0;
    JDOptions jo;
    jo.gmres = p.jcd_gmres;
    jo.mixed_floor = p.mixed_floor;
    jo.mixed_refine = p.mixed_refine;
    // ortho vectors of this step (ts_optimize.hpp:217-223, ss_optimize.hpp:104-109)
    DBuf<double> ovec;
    if (!ortho_rp.empty()) {
        const uint64_t nx = x.b.total;
        ovec.alloc(ortho_rp.size() * (nx ? nx : 1));
        for (std::size_t o = 0; o < ortho_rp.size(); ++o) make_ortho(o, ovec.get() + o * nx);
        jo.ortho = ovec.get();
        jo.n_ortho = int(ortho_rp.size());
        jo.ortho_ld = nx;
    }
    const double E = jacobi_davidson(c, plan, x.b.d.get(), p.jcd_tol, p.jcd_maxiter, iters, p.precision, &jo, &napply);
    QCM_CUDA(cudaStreamSynchronize(c.s));
    st.jd_s += now_s() - t1;
    st.hpsi_count += uint64_t(napply);
    st.hpsi_flops += double(napply) * plan.flops;
    if (p.precision != 0) {
        st.hpsi_count64 += uint64_t(jo.fp64_applies);  // the FP64 residual correction's applies
        st.hpsi_flops64 += double(jo.fp64_applies) * plan.flops;
    }
    last_iters = iters;
    return E;
}

void DevDMRG::step_prepare_site(StepState& S, int _site) {
    S.step = _site;
    step_sites(_site, S.lr, S.site1, S.site2);
    S.timing = std::getenv("QCM_SWEEP_TIMING") != nullptr;
    S.t0 = now_s();
    S.tt[0] = S.t0;
    bnd_use(left_[S.site1].get());
    bnd_use(right_[S.site2 + 1].get());
    make_left_paired(c, mps[S.site1]);
    make_right_paired(c, mps[S.site2]);
    S.tst = DTwoSite();
    S.pre_done = false;
    S.tst.build(c, mps[S.site1], mps[S.site2]);
    if (S.timing) {
        QCM_CUDA(cudaStreamSynchronize(c.s));
        S.tt[1] = now_s();
    }
}

void DevDMRG::step_prepare_plan(StepState& S) {
    S.resident = false;
    S.plan = plan_for(S.step, *left_[S.site1], *right_[S.site2 + 1], ts_mpo[S.site1], S.tst.phys, S.tst.twin.left,
                      S.tst.right, S.key, S.resident);
    S.plan->stream = c.s;
    S.tt[2] = now_s();
}

void DevDMRG::step_prepare_stage(StepState& S, bool group) {
    if (!S.resident && !group) {
        stream_coefficients(*S.plan, coefficient_budget);
        chunk_sectors(*S.plan, apply_budget);
    }
    if (group) {
        // applied only inside the step's plan group: its coefficient blocks, not its work lists
        if (!S.resident) upload_plan(*S.plan, false);
    } else if (S.resident) {
        restage_plan(*S.plan);
    } else {
        upload_plan(*S.plan);
    }
    QCM_CUDA(cudaStreamSynchronize(c.s));
    S.t1 = now_s();
}

void DevDMRG::step_prepare(StepState& S, int _site) {
    step_prepare_site(S, _site);
    step_prepare_plan(S);
    step_prepare_stage(S, false);
    st.plan_s += S.t1 - S.t0;
}

void DevDMRG::step_finish_pre(StepState& S) {
    if (S.pre_done) return;
    S.t2 = now_s();
    keep_plan(S.step, std::move(S.plan), S.key);
    S.tst.twin_to_both(c);
    if (S.timing) {
        QCM_CUDA(cudaStreamSynchronize(c.s));
        S.tt[3] = now_s();
    }
    S.pre_done = true;
}

void DevDMRG::step_finish(StepState& S, double E, double& energy, TruncResults& tr, const BlockSVD* sv, std::size_t b0,
                          std::size_t g) {
    const int _site = S.step, site1 = S.site1, site2 = S.site2;
    DTwoSite& tst = S.tst;
    auto mark = [&](int i) {
        if (!S.timing) return;
        QCM_CUDA(cudaStreamSynchronize(c.s));
        S.tt[i] = now_s();
    };
    step_finish_pre(S);
    const double t2 = S.t2;
    energy = E + p.ecore;
    double t3_last = 0;
    const double alpha = sweep_count < p.ngrowsweeps ? p.alpha_initial
                         : (sweep_count < p.ngrowsweeps + p.nmainsweeps ? p.alpha_main : p.alpha_final);
    if (S.lr == 1) {
        tr = p.heev ? tst.predict_split(c, true, p.Mmax, p.cutoff, alpha, *left_[site1], mpo[site1], mps[site1], mps[site2])
             : sv   ? tst.split_from(c, true, *sv, b0, g, mps[site1], mps[site2])
                    : tst.split(c, true, p.Mmax, p.cutoff, mps[site1], mps[site2]);
        mark(4);
        DBlocks t = normalize_left(c, mps[site2]);
        if (site2 < L - 1) multiply_from_left(c, mps[site2 + 1], t);
        QCM_CUDA(cudaStreamSynchronize(c.s));
        const double t3 = now_s();
        t3_last = t3;
        st.trunc_s += t3 - t2;
        DMPS ket = right_paired_copy(c, mps[site1]);
        left_[site2] = boundary_step_left(c, *left_[site1], ket, mps[site1], mpo[site1], true, bstep_cache_for(_site));
        bstep_cache_done(_site);
        for (std::size_t o = 0; o < ortho_rp.size(); ++o)
            ortho_left_[o][site2] = ortho_left_step(c, mps[site1], ortho_rp[o][site1], ortho_left_[o][site1]);
        QCM_CUDA(cudaStreamSynchronize(c.s));
        // the right-to-left half-sweep rebuilds every right boundary but the last: this one is done
        if (site2 + 1 < L) right_[site2 + 1].reset();
        if (site2 == L - 1) left_[site2].reset();  // no two-site step reads the last left boundary
        st.boundary_s += now_s() - t3;
    } else {
        tr = p.heev ? tst.predict_split(c, false, p.Mmax, p.cutoff, alpha, *right_[site2 + 1], mpo[site2], mps[site1], mps[site2])
             : sv   ? tst.split_from(c, false, *sv, b0, g, mps[site1], mps[site2])
                    : tst.split(c, false, p.Mmax, p.cutoff, mps[site1], mps[site2]);
        mark(4);
        DBlocks t = normalize_right(c, mps[site1]);
        if (site1 > 0) multiply_from_right(c, mps[site1 - 1], t);
        QCM_CUDA(cudaStreamSynchronize(c.s));
        const double t3 = now_s();
        t3_last = t3;
        st.trunc_s += t3 - t2;
        right_[site2] = boundary_step_right(c, *right_[site2 + 1], mps[site2], mpo[site2], true, bstep_cache_for(_site));
        bstep_cache_done(_site);
        for (std::size_t o = 0; o < ortho_rp.size(); ++o)
            ortho_right_[o][site2] = ortho_right_step(c, mps[site2], ortho_lp[o][site2], ortho_right_[o][site2 + 1]);
        QCM_CUDA(cudaStreamSynchronize(c.s));
        // the next left-to-right half-sweep rebuilds every left boundary but the first
        if (site1 > 0) left_[site1].reset();
        if (site2 == 1) right_[site2].reset();  // no two-site step reads the first right boundary
        st.boundary_s += now_s() - t3;
    }
    bnd_trim(_site + 1);
    if (S.timing) {
        const double tend = now_s();
        std::fprintf(stderr,
                     "[step %d] twosite %.4f plan %.4f upload %.4f jd %.4f (%d) t2b %.4f svd %.4f qr %.4f bstep %.4f total %.4f\n",
                     _site, S.tt[1] - S.tt[0], S.tt[2] - S.tt[1], S.t1 - S.tt[2], t2 - S.t1, last_iters, S.tt[3] - t2,
                     S.tt[4] - S.tt[3], t3_last - S.tt[4], tend - t3_last, tend - S.tt[0]);
    }
}

void DevDMRG::step(int _site, double& energy, TruncResults& tr) {
    StepState S;
    step_prepare(S, _site);
    const int site1 = S.site1, site2 = S.site2;
    const double E = solve(*S.plan, S.tst.twin, [&](std::size_t o, double* v) {
        DTwoSite tso;
        tso.build(c, ortho_lp[o][site1], ortho_rp[o][site2]);
        ortho_vector(c, S.tst.twin, tso.twin, ortho_left_[o][site1], ortho_right_[o][site2 + 1], v);
    });
    step_finish(S, E, energy, tr);
}

void dmrg_group_sweep(const std::vector<DevDMRG*>& runs, std::vector<std::vector<double>>& energies,
                      std::vector<std::vector<TruncResults>>& trunc) {
    if (runs.empty()) throw std::runtime_error("DMRG group: no runs");
    DevDMRG& r0 = *runs[0];
    const int n = r0.steps_per_sweep();
    for (const DevDMRG* d : runs) {
        if (d->p.single_site || d->p.precision != 0 || d->p.jcd_gmres != 0 || !d->ortho_rp.empty())
            throw std::runtime_error("DMRG group: two-site FP64 runs without GMRES or ortho states only");
        if (d->steps_per_sweep() != n || d->next_step != 0 || d->c.s != r0.c.s)
            throw std::runtime_error("DMRG group: the runs differ in length, position or stream");
        if (d->p.jcd_tol != r0.p.jcd_tol || d->p.jcd_maxiter != r0.p.jcd_maxiter || d->p.jcd_maxiter > 16)
            throw std::runtime_error("DMRG group: the runs differ in the JD tolerance or iteration limit (at most 16)");
        if (d->coefficient_budget || d->apply_budget)
            throw std::runtime_error("DMRG group: a run with streamed coefficient blocks or chunked applies");
    }
    const std::size_t nr = runs.size();
    energies.assign(nr, {});
    trunc.assign(nr, {});
    const double t_start = now_s();
    std::vector<StepState> S(nr);
    const bool timing = std::getenv("QCM_SWEEP_TIMING") != nullptr;
    for (int step = 0; step < n; ++step) {
        // the runs' two-site tensors, then their plans (host schedules, built or re-bound from the previous
        // sweep, one run per thread), then their coefficient blocks
        const double tp = now_s();
        for (std::size_t i = 0; i < nr; ++i) runs[i]->step_prepare_site(S[i], step);
        std::vector<std::string> err(nr);
#pragma omp parallel for schedule(dynamic, 1)
        for (long i = 0; i < long(nr); ++i) {
            try {
                runs[std::size_t(i)]->step_prepare_plan(S[std::size_t(i)]);
            } catch (const std::exception& e) {
                err[std::size_t(i)] = e.what();
            }
        }
        for (const std::string& e : err)
            if (!e.empty()) throw std::runtime_error(e);
        for (std::size_t i = 0; i < nr; ++i) runs[i]->step_prepare_stage(S[i], true);
        double tm = 0, tjd = 0;
        // one plan group, one lockstep Jacobi-Davidson over every run's two-site problem
        const double tj = now_s();
        for (DevDMRG* d : runs) d->st.plan_s += (tj - tp) / double(nr);
        std::vector<HeffPlan*> plans(nr);
        for (std::size_t i = 0; i < nr; ++i) plans[i] = S[i].plan.get();
        std::vector<uint64_t> xo, xn(nr);
        std::vector<double> ev;
        std::vector<int> iters;
        int applies = 0;
        {
            AllocStream scope(r0.c.s);
            auto g = merge_plans(plans, xo, r0.c.s);
            if (timing) { QCM_CUDA(cudaStreamSynchronize(r0.c.s)); tm = now_s(); }
            DBuf<double> X(g->x_len ? g->x_len : 1);
            QCM_CUDA(cudaMemsetAsync(X.get(), 0, (g->x_len ? g->x_len : 1) * sizeof(double), r0.c.s));
            for (std::size_t i = 0; i < nr; ++i) {
                xn[i] = S[i].plan->x_len;
                if (xn[i] != S[i].tst.twin.b.total) throw std::runtime_error("DMRG group: twin layout differs from its plan");
                if (xn[i])
                    QCM_CUDA(cudaMemcpyAsync(X.get() + xo[i], S[i].tst.twin.b.d.get(), xn[i] * sizeof(double),
                                             cudaMemcpyDeviceToDevice, r0.c.s));
            }
            jacobi_davidson_batched(*g, xo, xn, X.get(), r0.p.jcd_tol, r0.p.jcd_maxiter, ev, iters, true, &applies);
            if (timing) { QCM_CUDA(cudaStreamSynchronize(r0.c.s)); tjd = now_s(); }
            for (std::size_t i = 0; i < nr; ++i)
                if (xn[i])
                    QCM_CUDA(cudaMemcpyAsync(S[i].tst.twin.b.d.get(), X.get() + xo[i], xn[i] * sizeof(double),
                                             cudaMemcpyDeviceToDevice, r0.c.s));
            QCM_CUDA(cudaStreamSynchronize(r0.c.s));
        }
        const double dt = (now_s() - tj) / double(nr);
        for (std::size_t i = 0; i < nr; ++i) {
            DevDMRG& d = *runs[i];
            d.st.jd_s += dt;
            d.st.hpsi_count += uint64_t(applies);
            d.st.hpsi_flops += double(applies) * S[i].plan->flops;
            d.last_iters = iters[i];
        }
        // the truncations: every run's two-site blocks in one decomposition (one QR, one Jacobi and one
        // assembly launch), each run cut by its own bond dimension and cutoff (runs truncating by the
        // density matrix run their own)
        for (std::size_t i = 0; i < nr; ++i) runs[i]->step_finish_pre(S[i]);
        std::vector<std::size_t> svd_run;
        for (std::size_t i = 0; i < nr; ++i)
            if (!runs[i]->p.heev) svd_run.push_back(i);
        BlockSVD sv;
        std::vector<std::size_t> b0(nr, 0), gi(nr, 0);
        if (!svd_run.empty()) {
            const double ts = now_s();
            DBlocks all;
            std::vector<std::size_t> g0{0};
            std::vector<uint64_t> mm;
            std::vector<double> co;
            std::vector<uint64_t> base;
            for (std::size_t q = 0; q < svd_run.size(); ++q) {
                const DBlocks& b = S[svd_run[q]].tst.both;
                b0[svd_run[q]] = all.n();
                gi[svd_run[q]] = q;
                base.push_back(all.total);
                for (std::size_t k = 0; k < b.n(); ++k) {
                    all.lc.push_back(b.lc[k]); all.rc.push_back(b.rc[k]);
                    all.rows.push_back(b.rows[k]); all.cols.push_back(b.cols[k]);
                    all.off.push_back(all.total + b.off[k]);
                }
                all.total += (b.total + 31) / 32 * 32;
                g0.push_back(all.n());
                mm.push_back(runs[svd_run[q]]->p.Mmax);
                co.push_back(runs[svd_run[q]]->p.cutoff);
            }
            all.allocate(r0.c.s, false);
            for (std::size_t q = 0; q < svd_run.size(); ++q) {
                const DBlocks& b = S[svd_run[q]].tst.both;
                if (b.total)
                    QCM_CUDA(cudaMemcpyAsync(all.d.get() + base[q], b.d.get(), b.total * sizeof(double),
                                             cudaMemcpyDeviceToDevice, r0.c.s));
            }
            sv = svd_truncate_groups(r0.c, all, g0, mm, co);
            const double dts = (now_s() - ts) / double(svd_run.size());
            for (std::size_t i : svd_run) runs[i]->st.trunc_s += dts;
        }
        for (std::size_t i = 0; i < nr; ++i) {
            DevDMRG& d = *runs[i];
            double E = 0;
            TruncResults tr;
            S[i].t2 = now_s();  // the shared decomposition is counted above
            if (d.p.heev) d.step_finish(S[i], ev[i], E, tr);
            else d.step_finish(S[i], ev[i], E, tr, &sv, b0[i], gi[i]);
            energies[i].push_back(E);
            trunc[i].push_back(tr);
        }
        if (timing)
            std::fprintf(stderr, "[group step %d] prepare %.4f merge %.4f jd %.4f (%d applies) finish %.4f\n", step, tj - tp,
                         tm - tj, tjd - tm, applies, now_s() - tjd);
    }
    const double dt = (now_s() - t_start) / double(nr);
    for (DevDMRG* d : runs) {
        d->next_step = 0;
        ++d->sweep_count;
        d->st.total_s += dt;
    }
}

void DevDMRG::step_single(int _site, double& energy, TruncResults& tr) {
    // to_site (ss_optimize.hpp:57-62): sites 0 .. L-1 left to right, then L-1 .. 0
    const int lr = _site < L ? 1 : -1;
    const int site = _site < L ? _site : 2 * L - 1 - _site;
    const double t0 = now_s();
    bnd_use(left_[site].get());
    bnd_use(right_[site + 1].get());
    make_right_paired(c, mps[site]);
    DMPS x = packed_right(c, mps[site]);
    // solve_site_problem with the single-site MPO tensor (ss_optimize.hpp:120)
    uint64_t key = 0;
    bool resident = false;
    auto plan = plan_for(_site, *left_[site], *right_[site + 1], mpo[site], x.phys, x.left, x.right, key, resident);
    plan->stream = c.s;
    if (plan->x_len != x.b.total) throw std::runtime_error("DMRG: site tensor layout differs from the plan");
    if (resident) {
        restage_plan(*plan);
    } else {
        stream_coefficients(*plan, coefficient_budget);
        chunk_sectors(*plan, apply_budget);
        upload_plan(*plan);
    }
    QCM_CUDA(cudaStreamSynchronize(c.s));
    st.plan_s += now_s() - t0;
    const double E = solve(*plan, x, [&](std::size_t o, double* v) {
        ortho_vector(c, x, ortho_rp[o][site], ortho_left_[o][site], ortho_right_[o][site + 1], v);
    });
    keep_plan(_site, std::move(plan), key);
    mps[site] = std::move(x);
    energy = E + p.ecore;
    // alpha, cutoff and Mmax of this sweep (ss_optimize.hpp:143-155)
    const double alpha = sweep_count < p.ngrowsweeps ? p.alpha_initial
                         : (sweep_count < p.ngrowsweeps + p.nmainsweeps ? p.alpha_main : p.alpha_final);
    tr = TruncResults();
    const double t2 = now_s();
    if (lr == 1) {
        // ss_optimize.hpp:158-173
        if (site < L - 1) tr = grow_l2r(c, mps[site], mps[site + 1], *left_[site], mpo[site], alpha, p.Mmax, p.cutoff);
        else normalize_left(c, mps[site]);
        QCM_CUDA(cudaStreamSynchronize(c.s));
        const double t3 = now_s();
        st.trunc_s += t3 - t2;
        DMPS ket = right_paired_copy(c, mps[site]);
        left_[site + 1] = boundary_step_left(c, *left_[site], ket, mps[site], mpo[site], true, bstep_cache_for(_site));
        bstep_cache_done(_site);
        for (std::size_t o = 0; o < ortho_rp.size(); ++o)
            ortho_left_[o][site + 1] = ortho_left_step(c, mps[site], ortho_rp[o][site], ortho_left_[o][site]);
        QCM_CUDA(cudaStreamSynchronize(c.s));
        // the right-to-left half-sweep rebuilds every right boundary but the last; none reads left_[L]
        if (site + 1 < L) right_[site + 1].reset();
        else left_[site + 1].reset();
        st.boundary_s += now_s() - t3;
    } else {
        // ss_optimize.hpp:174-186
        if (site > 0) tr = grow_r2l(c, mps[site], mps[site - 1], *right_[site + 1], mpo[site], alpha, p.Mmax, p.cutoff);
        else normalize_right(c, mps[site]);
        QCM_CUDA(cudaStreamSynchronize(c.s));
        const double t3 = now_s();
        st.trunc_s += t3 - t2;
        right_[site] = boundary_step_right(c, *right_[site + 1], mps[site], mpo[site], true, bstep_cache_for(_site));
        bstep_cache_done(_site);
        for (std::size_t o = 0; o < ortho_rp.size(); ++o)
            ortho_right_[o][site] = ortho_right_step(c, mps[site], ortho_lp[o][site], ortho_right_[o][site + 1]);
        QCM_CUDA(cudaStreamSynchronize(c.s));
        // the next left-to-right half-sweep rebuilds every left boundary but the first; none reads right_[0]
        if (site > 0) left_[site].reset();
        else right_[site].reset();
        st.boundary_s += now_s() - t3;
    }
    bnd_trim(_site + 1);
}

void DevDMRG::run_until(int stop, std::vector<double>& energies, std::vector<TruncResults>& trunc) {
    const int n = steps_per_sweep();
    if (stop < next_step || stop > n) throw std::runtime_error("DMRG: stop step outside the current sweep");
    const double t_start = now_s();
    for (; next_step < stop; ++next_step) {
        double E = 0;
        TruncResults tr;
        if (p.single_site) step_single(next_step, E, tr);
        else step(next_step, E, tr);
        energies.push_back(E);
        trunc.push_back(tr);
    }
    if (next_step == n) { next_step = 0; ++sweep_count; }
    st.total_s += now_s() - t_start;
}

void DevDMRG::sweep(std::vector<double>& energies, std::vector<TruncResults>& trunc) {
    energies.clear();
    trunc.clear();
    run_until(steps_per_sweep(), energies, trunc);
}

void DevDMRG::pending_twin(std::vector<double>& twin) {
    if (p.single_site) throw std::runtime_error("DMRG: pending site problems of two-site sweeps only");
    int lr, site1, site2;
    step_sites(next_step, lr, site1, site2);
    bnd_use(left_[site1].get());
    bnd_use(right_[site2 + 1].get());
    make_left_paired(c, mps[site1]);
    make_right_paired(c, mps[site2]);
    DTwoSite tst;
    tst.build(c, mps[site1], mps[site2]);
    twin.resize(tst.twin.b.total);
    if (!twin.empty())
        QCM_CUDA(cudaMemcpyAsync(twin.data(), tst.twin.b.d.get(), twin.size() * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    QCM_CUDA(cudaStreamSynchronize(c.s));
}

std::unique_ptr<HeffPlan> DevDMRG::pending_plan(std::vector<double>* twin, Index* phys_out, Index* left_out,
                                                Index* right_out) {
    if (p.single_site) throw std::runtime_error("DMRG: pending site problems of two-site sweeps only");
    int lr, site1, site2;
    step_sites(next_step, lr, site1, site2);
    bnd_use(left_[site1].get());
    bnd_use(right_[site2 + 1].get());
    make_left_paired(c, mps[site1]);
    make_right_paired(c, mps[site2]);
    DTwoSite tst;
    tst.build(c, mps[site1], mps[site2]);
    auto plan = build_heff_plan(*left_[site1], *right_[site2 + 1], ts_mpo[site1], tst.phys, tst.twin.left, tst.right, false);
    plan->stream = c.s;
    if (twin) {
        twin->resize(plan->x_len);
        if (plan->x_len != tst.twin.b.total) throw std::runtime_error("DMRG: twin layout differs from the plan");
        QCM_CUDA(cudaMemcpyAsync(twin->data(), tst.twin.b.d.get(), plan->x_len * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    }
    QCM_CUDA(cudaStreamSynchronize(c.s));
    if (phys_out) *phys_out = tst.phys;
    if (left_out) *left_out = tst.twin.left;
    if (right_out) *right_out = tst.right;
    return plan;
}

}  // namespace qcm
