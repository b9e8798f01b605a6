// plan.cpp -- host side of the builder plan: basis, interpolation points, matrix assembly, banded
// factorisation and the device tables of the chunked sweeps.
//
// Everything here runs once per plan (the reference's SplineBuilder constructor,
// spline_builder.hpp:227-260). The factorisations are written from the published unblocked
// algorithms (Gaussian elimination with partial pivoting in band storage, Golub & Van Loan
// "Matrix Computations" 4.3.5; Gauss-Jordan for the small Schur block).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <map>

#include "ddcb_internal.hpp"

namespace ddcb {

namespace {

int n_boundary_equations(int bc, int degree)
{
    if (bc == DDCB_PERIODIC || bc == DDCB_GREVILLE) return 0;
    return degree / 2; // spline_builder_closures.hpp:43-55
}

double ipow(double a, int i)
{
    double r = 1.0;
    for (int j = 0; j < i; ++j) r *= a; // math_tools.hpp:67-75 (repeated product)
    return r;
}

long modulo(long x, long y) { return x - y * static_cast<long>(std::floor(double(x) / double(y))); }

} // namespace

// ---------------------------------------------------------------------------------------------
// Bases
// ---------------------------------------------------------------------------------------------
void make_uniform_basis(Basis& b, int degree, bool periodic, double rmin, double rmax, long ncells)
{
    if (degree < 1 || degree > 5) throw Error(DDCB_ERR_UNSUPPORTED, "degree must be in 1..5");
    if (ncells < 1) throw Error(DDCB_ERR_INVALID_ARGUMENT, "ncells must be positive");
    if (!(rmin < rmax)) throw Error(DDCB_ERR_INVALID_ARGUMENT, "rmin must be below rmax");
    if (ncells > (1L << 24)) throw Error(DDCB_ERR_UNSUPPORTED, "ncells too large");
    // Ghosted uniform knots: step = (rmax-rmin)/ncells, knot k at origin + k*step with
    // origin = rmin - degree*step (uniform_point_sampling.hpp:170-192, bsplines_uniform.hpp:145).
    double const step = (rmax - rmin) / double(ncells);
    double const origin = rmin - double(degree) * step;
    BasisDesc& d = b.desc;
    d.degree = degree;
    d.periodic = periodic;
    d.uniform = 1;
    d.ncells = int(ncells);
    d.step = step;
    d.inv_step = 1.0 / step;
    d.rmin = origin + double(degree) * step;
    d.rmax = origin + double(degree + ncells) * step;
    d.length = d.rmax - d.rmin;
    b.knots.resize(ncells + 1 + 2 * degree);
    for (size_t k = 0; k < b.knots.size(); ++k) b.knots[k] = origin + double(k) * step;
    d.knots = b.knots.data();
}

void make_non_uniform_basis(Basis& b, int degree, bool periodic, double const* breaks, long nbreaks)
{
    if (degree < 1 || degree > 5) throw Error(DDCB_ERR_UNSUPPORTED, "degree must be in 1..5");
    if (nbreaks < 2 || breaks == nullptr) throw Error(DDCB_ERR_INVALID_ARGUMENT, "at least two break points are needed");
    if (nbreaks > (1L << 24)) throw Error(DDCB_ERR_UNSUPPORTED, "too many break points");
    for (long i = 1; i < nbreaks; ++i)
        if (!(breaks[i] > breaks[i - 1])) throw Error(DDCB_ERR_INVALID_ARGUMENT, "break points must be strictly increasing");
    long const nc = nbreaks - 1;
    std::vector<double>& k = b.knots;
    k.assign(nbreaks + 2 * degree, 0.0);
    for (long i = 0; i < nbreaks; ++i) k[degree + i] = breaks[i];
    double const rmin = k[degree], rmax = k[degree + nc];
    // Periodic: knots continued by the period; otherwise clamped (bsplines_non_uniform.hpp:437-455).
    if (periodic) {
        double const period = rmax - rmin;
        for (int i = 1; i < degree + 1; ++i) {
            k[degree - i] = k[degree + nc - i] - period;
            k[degree + nc + i] = k[degree + i] + period;
        }
    } else {
        for (int i = 1; i < degree + 1; ++i) {
            k[degree - i] = rmin;
            k[degree + nc + i] = rmax;
        }
    }
    BasisDesc& d = b.desc;
    d.degree = degree;
    d.periodic = periodic;
    d.uniform = 0;
    d.ncells = int(nc);
    d.rmin = rmin;
    d.rmax = rmax;
    d.length = rmax - rmin;
    d.step = (rmax - rmin) / double(nc);
    d.inv_step = 1.0 / d.step;
    d.knots = k.data();
}

void upload_basis(Basis& b, int device)
{
    if (b.d_knots && b.device == device) return;
    free_basis(b);
    DDCB_CUDA_CHECK(cudaMalloc(&b.d_knots, b.knots.size() * sizeof(double)));
    DDCB_CUDA_CHECK(cudaMemcpy(b.d_knots, b.knots.data(), b.knots.size() * sizeof(double), cudaMemcpyHostToDevice));
    b.device = device;
}

void free_basis(Basis& b)
{
    if (b.d_knots) cudaFree(b.d_knots);
    b.d_knots = nullptr;
    b.device = -1;
}

// Integrals of the B-splines over [rmin, rmax] (integrals.hpp:30-153), size() entries.
void basis_integrals(Basis const& b, double* out)
{
    BasisDesc const& d = b.desc;
    long const sz = b.size(), nb = b.nbasis();
    if (d.uniform) {
        if (d.periodic) {
            for (long i = 0; i < nb; ++i) out[i] = d.step;
            for (long i = nb; i < sz; ++i) out[i] = 0.0;
            return;
        }
        for (long i = d.degree; i < sz - d.degree; ++i) out[i] = d.step;
        // Edge B-splines: step * (1 - partial sums of the degree+1 basis at rmin).
        double v[kMaxDegree + 2];
        double offset;
        uniform_cell(d, d.rmin, offset);
        uniform_values(d.degree + 1, offset, v);
        double total = 0.0;
        for (int i = 0; i < d.degree + 2; ++i) total += v[i];
        for (int i = 0; i < d.degree; ++i) {
            double part = 0.0;
            for (int j = 0; j < d.degree - i; ++j) part += v[j];
            out[i] = d.step * (total - part);
            out[sz - 1 - i] = d.step * (total - part);
        }
        return;
    }
    double const inv = 1.0 / (d.degree + 1);
    for (long i = 0; i < nb; ++i) out[i] = (b.knots[i + d.degree + 1] - b.knots[i]) * inv;
    for (long i = nb; i < sz; ++i) out[i] = 0.0;
}

// GrevilleInterpolationPoints (greville_interpolation_points.hpp:47-269).
std::vector<double> greville_points(Basis const& b, int lo, int hi)
{
    BasisDesc const& D = b.desc;
    int const d = D.degree;
    if ((lo == DDCB_PERIODIC) != (D.periodic != 0) || (hi == DDCB_PERIODIC) != (D.periodic != 0))
        throw Error(DDCB_ERR_INVALID_ARGUMENT, "closures do not match the periodicity of the basis");
    int const n_lo = n_boundary_equations(lo, d), n_hi = n_boundary_equations(hi, d);
    long const nb = b.nbasis();
    long const npts = nb - n_lo - n_hi;
    std::vector<double> pts(npts);
    if (D.uniform) {
        double const shift = (d % 2 == 0) ? 0.5 : 0.0;
        double const dx = (D.rmax - D.rmin) / double(D.ncells);
        double const o = D.rmin + shift * dx;
        if (D.periodic || (n_lo && n_hi)) {
            for (long i = 0; i < npts; ++i) pts[i] = o + double(i) * dx;
            return pts;
        }
        if (lo == DDCB_GREVILLE) {
            for (int i = 0; i < d / 2 + 1; ++i) {
                double s = (d - i) * D.rmin;
                long const last = i + d + 1; // last support knot of B-spline i
                for (long k = last - i; k < last; ++k) s += b.knots[k];
                pts[i] = s / d;
            }
        } else {
            pts[0] = o;
        }
        long const n_start = (lo == DDCB_GREVILLE) ? d / 2 + 1 : 1;
        for (long ip = 1; ip < D.ncells; ++ip) pts[ip - 1 + n_start] = o + double(ip) * dx;
        if (hi == DDCB_GREVILLE) {
            for (int i = 0; i < d / 2 + 1; ++i) {
                double s = (d - i) * D.rmax;
                long const first = nb - 1 - i + 1; // first support knot of B-spline nb-1-i, plus one
                for (long k = first; k < first + i; ++k) s += b.knots[k];
                pts[npts - 1 - i] = s / d;
            }
        } else {
            pts[npts - 1] = o + double(D.ncells - 1 + d % 2) * dx;
        }
        return pts;
    }
    std::vector<double> g(nb);
    for (long ib = 0; ib < nb; ++ib) {
        double s = 0.0;
        for (long k = ib + 1; k < ib + 1 + d; ++k) s += b.knots[k];
        g[ib] = s / d;
    }
    if (D.periodic) {
        // rotate the points that fall below rmin to the end (greville_interpolation_points.hpp:104-126)
        long np = 0;
        std::vector<double> tmp;
        while (np < nb && g[np] < D.rmin) {
            tmp.push_back(g[np] + D.length);
            ++np;
        }
        std::vector<double> r(g.begin() + np, g.end());
        r.insert(r.end(), tmp.begin(), tmp.end());
        std::copy(r.begin(), r.begin() + npts, pts.begin());
        return pts;
    }
    for (long i = 0; i < npts; ++i) pts[i] = g[i + n_lo];
    return pts;
}

// ---------------------------------------------------------------------------------------------
// Banded LU with partial pivoting (band storage of width 2kl+ku+1, as LAPACK's xGBTRF layout)
// ---------------------------------------------------------------------------------------------
namespace {

struct BandLU
{
    long m = 0, kl = 0, ku = 0;
    std::vector<double> w; // (2kl+ku+1) x m ; element (i,j) at w[(kl+ku+i-j)*m + j]
    std::vector<int> ipiv;
    double& at(long i, long j) { return w[(kl + ku + i - j) * m + j]; }
    double at(long i, long j) const { return w[(kl + ku + i - j) * m + j]; }

    void factor()
    {
        ipiv.assign(m, 0);
        long ju = 0;
        for (long j = 0; j < m; ++j) {
            long const km = std::min(kl, m - 1 - j);
            long jp = 0;
            double amax = std::fabs(at(j, j));
            for (long t = 1; t <= km; ++t)
                if (std::fabs(at(j + t, j)) > amax) {
                    amax = std::fabs(at(j + t, j));
                    jp = t;
                }
            ipiv[j] = int(j + jp);
            if (at(j + jp, j) == 0.0) throw Error(DDCB_ERR_SINGULAR, "singular interpolation matrix (zero pivot at row " + std::to_string(j) + ")");
            ju = std::max(ju, std::min(j + ku + jp, m - 1));
            if (jp != 0)
                for (long c = j; c <= ju; ++c) std::swap(at(j, c), at(j + jp, c));
            if (km > 0) {
                double const inv = 1.0 / at(j, j);
                for (long t = 1; t <= km; ++t) at(j + t, j) *= inv;
                for (long c = j + 1; c <= ju; ++c) {
                    double const u = at(j, c);
                    if (u != 0.0)
                        for (long t = 1; t <= km; ++t) at(j + t, c) -= at(j + t, j) * u;
                }
            }
        }
    }

    // x <- Q^-1 x (or Q^-T x), one column
    void solve(double* x, bool transpose) const
    {
        long const kv = kl + ku;
        if (!transpose) {
            for (long j = 0; j < m; ++j) {
                long const l = ipiv[j];
                if (l != j) std::swap(x[l], x[j]);
                long const lm = std::min(kl, m - 1 - j);
                for (long t = 1; t <= lm; ++t) x[j + t] -= at(j + t, j) * x[j];
            }
            for (long j = m - 1; j >= 0; --j) {
                double s = x[j];
                for (long t = 1; t <= kv && j + t < m; ++t) s -= at(j, j + t) * x[j + t];
                x[j] = s / at(j, j);
            }
        } else {
            for (long j = 0; j < m; ++j) {
                double s = x[j];
                for (long t = 1; t <= kv && j - t >= 0; ++t) s -= at(j - t, j) * x[j - t];
                x[j] = s / at(j, j);
            }
            for (long j = m - 1; j >= 0; --j) {
                long const lm = std::min(kl, m - 1 - j);
                for (long t = 1; t <= lm; ++t) x[j] -= at(j + t, j) * x[j + t];
                long const l = ipiv[j];
                if (l != j) std::swap(x[l], x[j]);
            }
        }
    }
};

// Gauss-Jordan inverse with partial pivoting of a small dense matrix (row-major k x k).
std::vector<double> small_inverse(std::vector<double> a, long k)
{
    std::vector<double> inv(k * k, 0.0);
    for (long i = 0; i < k; ++i) inv[i * k + i] = 1.0;
    for (long c = 0; c < k; ++c) {
        long p = c;
        for (long r = c + 1; r < k; ++r)
            if (std::fabs(a[r * k + c]) > std::fabs(a[p * k + c])) p = r;
        if (a[p * k + c] == 0.0) throw Error(DDCB_ERR_SINGULAR, "singular Schur complement of the border block");
        if (p != c)
            for (long j = 0; j < k; ++j) {
                std::swap(a[p * k + j], a[c * k + j]);
                std::swap(inv[p * k + j], inv[c * k + j]);
            }
        double const piv = a[c * k + c];
        for (long j = 0; j < k; ++j) {
            a[c * k + j] /= piv;
            inv[c * k + j] /= piv;
        }
        for (long r = 0; r < k; ++r) {
            if (r == c) continue;
            double const f = a[r * k + c];
            if (f == 0.0) continue;
            for (long j = 0; j < k; ++j) {
                a[r * k + j] -= f * a[c * k + j];
                inv[r * k + j] -= f * inv[c * k + j];
            }
        }
    }
    return inv;
}

// Sparse rows of the assembled matrix: row -> (col -> value)
using SparseRows = std::vector<std::map<long, double>>;

// Host form of the device solve: border split, band LU of Q, Schur inverse and chunk transfers.
struct HostSolve
{
    long n = 0, m = 0, k = 0;
    BandLU lu;
    std::vector<double> gam;   // m x k (gamma, then Q^-1 gamma)
    std::vector<double> lam;   // k x m
    std::vector<double> Sinv;  // k x k
    long kl = 0, ku = 0;       // effective L / U bandwidths
    bool pivot = false;
    // chunking
    long nchunk = 1, chunk_len = 0;
    std::vector<double> Lf, Uf, PhiF, PhiB;
    std::vector<int8_t> piv;
    long qg_lo = 0, qg_hi = 0;
    std::vector<double> qg_rows;
    std::vector<int> lam_row, lam_col;
    std::vector<double> lam_val;

    long chunk_begin(long c) const { return c * chunk_len; }
    long chunk_end(long c) const { return (c == nchunk - 1) ? m : (c + 1) * chunk_len; }

    void analyse(SparseRows const& rows, bool periodic)
    {
        n = long(rows.size());
        // Border: periodic systems couple the ends; the circular bandwidth sets the border size.
        k = 0;
        if (periodic) {
            long bl = 0, bu = 0;
            for (long i = 0; i < n; ++i)
                for (auto const& [j, v] : rows[i]) {
                    if (v == 0.0) continue;
                    long o = modulo(j - i, n);
                    if (o > n / 2) o -= n;
                    bl = std::max(bl, -o);
                    bu = std::max(bu, o);
                }
            k = std::max(bl, bu);
        }
        if (n <= 16 || n <= 4 * k + 4) k = n; // tiny systems: all border (dense)
        m = n - k;
        long klq = 0, kuq = 0;
        for (long i = 0; i < m; ++i)
            for (auto const& [j, v] : rows[i])
                if (j < m && v != 0.0) {
                    klq = std::max(klq, i - j);
                    kuq = std::max(kuq, j - i);
                }
        lu.m = m;
        lu.kl = klq;
        lu.ku = kuq;
        lu.w.assign((2 * klq + kuq + 1) * std::max<long>(m, 1), 0.0);
        gam.assign(m * k, 0.0);
        lam.assign(k * m, 0.0);
        std::vector<double> delta(k * k, 0.0);
        for (long i = 0; i < n; ++i)
            for (auto const& [j, v] : rows[i]) {
                if (v == 0.0) continue; // explicit zeros may lie outside the band
                if (i < m && j < m) lu.at(i, j) = v;
                else if (i < m) gam[i * k + (j - m)] = v;
                else if (j < m) lam[(i - m) * m + j] = v;
                else delta[(i - m) * k + (j - m)] = v;
            }
        if (m > 0) lu.factor();
        // Q^-1 gamma
        std::vector<double> col(m);
        for (long r = 0; r < k; ++r) {
            for (long i = 0; i < m; ++i) col[i] = gam[i * k + r];
            if (m > 0) lu.solve(col.data(), false);
            for (long i = 0; i < m; ++i) gam[i * k + r] = col[i];
        }
        // Schur complement S = delta - lambda Q^-1 gamma
        std::vector<double> S = delta;
        for (long i = 0; i < k; ++i)
            for (long j = 0; j < k; ++j) {
                double s = 0.0;
                for (long l = 0; l < m; ++l) s += lam[i * m + l] * gam[l * k + j];
                S[i * k + j] -= s;
            }
        Sinv = k ? small_inverse(S, k) : std::vector<double>();
        // effective bandwidths of the factors
        kl = lu.kl;
        ku = 0;
        pivot = false;
        for (long j = 0; j < m; ++j) {
            if (lu.ipiv[j] != j) pivot = true;
            for (long t = 1; t <= lu.kl + lu.ku && j + t < m; ++t)
                if (lu.at(j, j + t) != 0.0) ku = std::max(ku, t);
        }
        // pad the bandwidths up to the shapes the kernels are compiled for (build_kernels.cu)
        auto up = [](long v, std::initializer_list<long> menu) {
            for (long x : menu)
                if (v <= x) return x;
            return -1L;
        };
        long const klp = up(std::max(kl, 1L), {1, 2, 4});
        long kup = up(std::max(ku, 1L), {1, 2, 4, 8});
        if (klp < 0 || kup < 0)
            throw Error(DDCB_ERR_UNSUPPORTED, "band too wide for the device solver (kl=" + std::to_string(kl) + ", ku=" + std::to_string(ku) + ")");
        kl = klp;
        ku = std::max(kup, klp);
        // lambda in COO form
        for (long i = 0; i < k; ++i)
            for (long j = 0; j < m; ++j)
                if (lam[i * m + j] != 0.0) {
                    lam_row.push_back(int(i));
                    lam_col.push_back(int(j));
                    lam_val.push_back(lam[i * m + j]);
                }
        // rows of Q^-1 gamma that matter (the correction decays away from the ends)
        double gmax = 0.0;
        for (double v : gam) gmax = std::max(gmax, std::fabs(v));
        double const thr = 1e-19 * gmax;
        auto row_big = [&](long i) {
            for (long r = 0; r < k; ++r)
                if (std::fabs(gam[i * k + r]) > thr) return true;
            return false;
        };
        long lo_end = 0, hi_begin = m;
        for (long i = 0; i < m; ++i)
            if (row_big(i)) lo_end = i + 1;
            else if (i > 2 * k + 8) break;
        for (long i = m - 1; i >= 0; --i)
            if (row_big(i)) hi_begin = i;
            else if (m - 1 - i > 2 * k + 8) break;
        if (hi_begin <= lo_end) {
            qg_lo = m;
            qg_hi = 0;
        } else {
            qg_lo = lo_end;
            qg_hi = m - hi_begin;
        }
        if (k == 0) qg_lo = qg_hi = 0;
        qg_rows.clear();
        for (long i = 0; i < qg_lo; ++i)
            for (long r = 0; r < k; ++r) qg_rows.push_back(gam[i * k + r]);
        for (long i = m - qg_hi; i < m; ++i)
            for (long r = 0; r < k; ++r) qg_rows.push_back(gam[i * k + r]);
    }

    // Forward step semantics shared with the kernel (build_kernels.cu, fwd_steps): window w holds
    // rows j..j+kl; swap, emit w[0], eliminate, shift.
    void fwd_steps(long a, long e, double* w /* kl entries */) const
    {
        std::vector<double> win(kl + 1);
        for (long t = 0; t < kl; ++t) win[t] = w[t];
        for (long j = a; j < e; ++j) {
            win[kl] = 0.0;
            long const p = piv[j];
            if (p) std::swap(win[0], win[p]);
            double const y = win[0];
            for (long t = 1; t <= kl; ++t) win[t] -= Lf[j * kl + t - 1] * y;
            for (long t = 0; t < kl; ++t) win[t] = win[t + 1];
        }
        for (long t = 0; t < kl; ++t) w[t] = win[t];
    }

    void bwd_steps(long a, long e, double* z /* ku entries */) const
    {
        for (long j = e - 1; j >= a; --j) {
            double s = 0.0;
            for (long t = 1; t <= ku; ++t) s -= Uf[j * (ku + 1) + t] * z[t - 1];
            double const x = s * Uf[j * (ku + 1)];
            for (long t = ku - 1; t >= 1; --t) z[t] = z[t - 1];
            if (ku > 0) z[0] = x;
        }
    }

    void make_tables(long nchunk_req)
    {
        // factor arrays in the kernel's layout
        Lf.assign(std::max<long>(m * kl, 1), 0.0);
        piv.assign(std::max<long>(m, 1), 0);
        Uf.assign(std::max<long>(m * (ku + 1), 1), 0.0);
        for (long j = 0; j < m; ++j) {
            piv[j] = int8_t(lu.ipiv[j] - j);
            for (long t = 1; t <= kl; ++t) Lf[j * kl + t - 1] = (t <= lu.kl && j + t < m) ? lu.at(j + t, j) : 0.0;
            Uf[j * (ku + 1)] = 1.0 / lu.at(j, j);
            for (long t = 1; t <= ku; ++t) Uf[j * (ku + 1) + t] = (t <= lu.kl + lu.ku && j + t < m) ? lu.at(j, j + t) : 0.0;
        }
        // chunking: odd chunk length (conflict-free shared-memory rows), at least max(kl,ku)+1 rows
        long const minlen = std::max<long>(std::max(kl, ku) + 1, 3);
        if (m == 0) {
            nchunk = 1;
            chunk_len = 0;
        } else {
            long L = (m + nchunk_req - 1) / std::max<long>(nchunk_req, 1);
            L = std::max(L, minlen);
            if (L % 2 == 0) L += 1;
            nchunk = std::max<long>(1, m / L);
            if (nchunk == 1) L = m;
            chunk_len = L;
        }
        PhiF.assign(std::max<long>(nchunk * kl * kl, 1), 0.0);
        PhiB.assign(std::max<long>(nchunk * ku * ku, 1), 0.0);
        std::vector<double> w(std::max<long>(kl, 1)), z(std::max<long>(ku, 1));
        for (long c = 0; c < nchunk && m > 0; ++c) {
            long const a = chunk_begin(c), e = chunk_end(c);
            for (long s = 0; s < kl; ++s) {
                std::fill(w.begin(), w.end(), 0.0);
                w[s] = 1.0;
                fwd_steps(a, e, w.data());
                for (long r = 0; r < kl; ++r) PhiF[(c * kl + r) * kl + s] = w[r];
            }
            for (long s = 0; s < ku; ++s) {
                std::fill(z.begin(), z.end(), 0.0);
                z[s] = 1.0;
                bwd_steps(a, e, z.data());
                for (long r = 0; r < ku; ++r) PhiB[(c * ku + r) * ku + s] = z[r];
            }
        }
    }

    // Full host solve of A x = rhs (or A^T x = rhs): used for quadrature coefficients.
    void solve_host(double* x, bool transpose) const
    {
        std::vector<double> x1(x, x + m), x2(x + m, x + n);
        if (!transpose) {
            if (m > 0) lu.solve(x1.data(), false);
            for (long i = 0; i < k; ++i) {
                double s = x2[i];
                for (long j = 0; j < m; ++j) s -= lam[i * m + j] * x1[j];
                x2[i] = s;
            }
            std::vector<double> y(k, 0.0);
            for (long i = 0; i < k; ++i)
                for (long j = 0; j < k; ++j) y[i] += Sinv[i * k + j] * x2[j];
            for (long i = 0; i < m; ++i)
                for (long r = 0; r < k; ++r) x1[i] -= gam[i * k + r] * y[r];
            std::copy(x1.begin(), x1.end(), x);
            std::copy(y.begin(), y.end(), x + m);
        } else {
            // A^T = [[Q^T, l^T],[g^T, S0^T]]; with g' = Q^-1 g: x1' = Q^-T r1,
            // x2 = S^-T (r2 - g'^T r1), x1 = Q^-T (r1 - l^T x2)
            std::vector<double> r2(k);
            for (long i = 0; i < k; ++i) {
                double s = x2[i];
                for (long j = 0; j < m; ++j) s -= gam[j * k + i] * x1[j];
                r2[i] = s;
            }
            std::vector<double> y(k, 0.0);
            for (long i = 0; i < k; ++i)
                for (long j = 0; j < k; ++j) y[i] += Sinv[j * k + i] * r2[j];
            for (long j = 0; j < m; ++j) {
                double s = x1[j];
                for (long i = 0; i < k; ++i) s -= lam[i * m + j] * y[i];
                x1[j] = s;
            }
            if (m > 0) lu.solve(x1.data(), true);
            std::copy(x1.begin(), x1.end(), x);
            std::copy(y.begin(), y.end(), x + m);
        }
    }
};

// The assembled interpolation matrix (spline_builder.hpp:784-886) as sparse rows.
SparseRows assemble(Builder const& bl)
{
    BasisDesc const& D = bl.basis.desc;
    int const d = D.degree;
    long const nb = bl.n;
    SparseRows rows(nb);
    int const nc = d / 2 + 1;
    auto hermite_rows = [&](double x, int nbe, bool upper) {
        double dv[(kMaxDegree + 1) * (kMaxDegree / 2 + 2)];
        eval_basis_and_n_derivs(D, x, nbe, dv);
        // dv is (d+1) x (nbe+1); scale derivative columns by dx^j (spline_builder.hpp:802-808)
        for (int i = 0; i < d + 1; ++i)
            for (int j = 1; j <= nbe && j < nc; ++j) dv[i * (nbe + 1) + j] *= ipow(bl.dx, j);
        for (int i = 0; i < nbe; ++i)
            for (int j = 0; j < d; ++j) {
                int const basis_j = upper ? j + 1 : j;
                double const v = dv[basis_j * (nbe + 1) + i + bl.odd];
                long const row = upper ? nb - nbe + i : i;
                long const colj = upper ? nb - d + j : j;
                rows[row][colj] = v;
            }
    };
    if (bl.lo == DDCB_HERMITE || bl.lo == DDCB_HOMOGENEOUS_HERMITE) hermite_rows(D.rmin, bl.nbe_lo, false);
    double v[kMaxDegree + 1];
    for (size_t ix = 0; ix < bl.points.size(); ++ix) {
        int const jmin = eval_basis(D, bl.points[ix], v);
        for (int s = 0; s < d + 1; ++s) {
            // Values below 1e-15 (a point a rounding error away from a knot) are dropped: the
            // reference's band storage keeps only its fixed band and discards such entries
            // (splines_linear_problem_band.cpp:95-97), so they never reach its solve either.
            if (std::fabs(v[s]) < 1e-15) continue;
            long const j = modulo(long(jmin) - bl.offset + s, nb);
            rows[long(ix) + bl.nbe_lo][j] = v[s];
        }
    }
    if (bl.hi == DDCB_HERMITE || bl.hi == DDCB_HOMOGENEOUS_HERMITE) hermite_rows(D.rmax, bl.nbe_hi, true);
    return rows;
}

SparseRows transpose_rows(SparseRows const& r)
{
    SparseRows t(r.size());
    for (size_t i = 0; i < r.size(); ++i)
        for (auto const& [j, v] : r[i]) t[j][long(i)] = v;
    return t;
}

// Device copy of a HostSolve; returns the SolveTables with device pointers into `block`.
SolveTables upload_tables(HostSolve const& h, std::vector<char>& blob, std::vector<size_t>& offs)
{
    SolveTables t {};
    t.n = int(h.n);
    t.m = int(h.m);
    t.k = int(h.k);
    t.kl = int(h.kl);
    t.ku = int(h.ku);
    t.pivot = h.pivot ? 1 : 0;
    t.nchunk = int(h.nchunk);
    t.chunk_len = int(h.chunk_len);
    t.lam_nnz = int(h.lam_val.size());
    t.qg_lo = int(h.qg_lo);
    t.qg_hi = int(h.qg_hi);
    auto push = [&](void const* p, size_t bytes) {
        size_t const off = (blob.size() + 255) / 256 * 256;
        blob.resize(off + std::max<size_t>(bytes, 8), 0);
        if (bytes) std::memcpy(blob.data() + off, p, bytes);
        offs.push_back(off);
        return off;
    };
    push(h.Lf.data(), h.Lf.size() * 8);
    push(h.piv.data(), h.piv.size());
    push(h.Uf.data(), h.Uf.size() * 8);
    push(h.PhiF.data(), h.PhiF.size() * 8);
    push(h.PhiB.data(), h.PhiB.size() * 8);
    push(h.lam_row.data(), h.lam_row.size() * 4);
    push(h.lam_col.data(), h.lam_col.size() * 4);
    push(h.lam_val.data(), h.lam_val.size() * 8);
    push(h.Sinv.data(), h.Sinv.size() * 8);
    push(h.qg_rows.data(), h.qg_rows.size() * 8);
    return t;
}

void bind_tables(SolveTables& t, char* base, size_t const* offs)
{
    t.Lf = reinterpret_cast<double const*>(base + offs[0]);
    t.piv = reinterpret_cast<int8_t const*>(base + offs[1]);
    t.Uf = reinterpret_cast<double const*>(base + offs[2]);
    t.PhiF = reinterpret_cast<double const*>(base + offs[3]);
    t.PhiB = reinterpret_cast<double const*>(base + offs[4]);
    t.lam_row = reinterpret_cast<int const*>(base + offs[5]);
    t.lam_col = reinterpret_cast<int const*>(base + offs[6]);
    t.lam_val = reinterpret_cast<double const*>(base + offs[7]);
    t.Sinv = reinterpret_cast<double const*>(base + offs[8]);
    t.Qg = reinterpret_cast<double const*>(base + offs[9]);
}

std::string describe(HostSolve const& h)
{
    return "border=" + std::to_string(h.k) + ",Q=BandLU(" + std::to_string(h.m) + ",kl=" + std::to_string(h.kl)
           + ",ku=" + std::to_string(h.ku) + (h.pivot ? ",pivoting" : "") + "),chunks=" + std::to_string(h.nchunk)
           + "x" + std::to_string(h.chunk_len);
}

} // namespace

// spline_builder.hpp:1244-1317
static void check_valid_grid(Builder const& b)
{
    BasisDesc const& D = b.basis.desc;
    long const expected = b.n - b.nbe_lo - b.nbe_hi;
    if (long(b.points.size()) != expected)
        throw Error(DDCB_ERR_BAD_GRID, "Incorrect number of points supplied to NonUniformInterpolationPoints. (Received : "
                                           + std::to_string(b.points.size()) + ", expected : " + std::to_string(expected));
    int in_cell = 0;
    long cell_end = D.degree + 1;
    auto check = [&](int npc, long cend) {
        if (npc > D.degree + 1)
            throw Error(DDCB_ERR_BAD_GRID, "The spline problem is overconstrained. There are " + std::to_string(npc)
                                               + " points in the " + std::to_string(cend - D.degree) + "-th cell.");
    };
    for (double p : b.points) {
        double const ce = b.basis.knots[cell_end];
        if (p > ce) {
            check(in_cell, cell_end);
            in_cell = 1;
            cell_end += 1;
        } else if (p == ce) {
            check(in_cell + 1, cell_end);
            in_cell = 1;
            cell_end += 1;
        } else {
            in_cell += 1;
        }
    }
    check(in_cell, cell_end);
}

struct BuilderPrivate
{
    HostSolve fwd, adj;
};

Builder* create_builder(Basis const& basis, double const* pts, long npts, int lo, int hi, ddcb_builder_options const* opts)
{
    if (pts == nullptr && npts > 0) throw Error(DDCB_ERR_INVALID_ARGUMENT, "interpolation points pointer is NULL");
    if (lo < 0 || lo > 3 || hi < 0 || hi > 3) throw Error(DDCB_ERR_INVALID_ARGUMENT, "unknown closure");
    if ((lo == DDCB_PERIODIC) != (hi == DDCB_PERIODIC)) throw Error(DDCB_ERR_INVALID_ARGUMENT, "Incompatible closure relations");
    if ((lo == DDCB_PERIODIC) != (basis.desc.periodic != 0))
        throw Error(DDCB_ERR_INVALID_ARGUMENT, "closure relations do not match the periodicity of the basis");
    auto* b = new Builder();
    try {
        b->basis.desc = basis.desc;
        b->basis.knots = basis.knots;
        b->basis.desc.knots = b->basis.knots.data();
        BasisDesc const& D = b->basis.desc;
        int const d = D.degree;
        b->lo = lo;
        b->hi = hi;
        b->nbe_lo = n_boundary_equations(lo, d);
        b->nbe_hi = n_boundary_equations(hi, d);
        b->nbv_lo = (lo == DDCB_HOMOGENEOUS_HERMITE) ? 0 : b->nbe_lo;
        b->nbv_hi = (hi == DDCB_HOMOGENEOUS_HERMITE) ? 0 : b->nbe_hi;
        b->odd = d % 2;
        b->dx = (D.rmax - D.rmin) / double(D.ncells);
        b->n = b->basis.nbasis();
        b->points.assign(pts, pts + npts);
        if (opts) {
            if (opts->precision != DDCB_FP64 && opts->precision != DDCB_FP32_REFINE)
                throw Error(DDCB_ERR_INVALID_ARGUMENT, "unknown precision");
            b->precision = opts->precision;
            if (opts->refine_rounds > 0) b->refine_rounds = std::min(opts->refine_rounds, 3);
            if (opts->tile_lines > 0) b->tile_lines = opts->tile_lines;
            if (opts->chunks > 0) b->nchunk_req = opts->chunks;
        }
        if (b->tile_lines != 1 && b->tile_lines != 4 && b->tile_lines != 8)
            throw Error(DDCB_ERR_INVALID_ARGUMENT, "tile_lines must be 1, 4 or 8");
        if (b->nchunk_req * b->tile_lines > 1024) throw Error(DDCB_ERR_INVALID_ARGUMENT, "tile_lines*chunks must be <= 1024");
        check_valid_grid(*b);
        // compute_offset (spline_builder.hpp:619-658)
        b->offset = 0;
        if (D.periodic) {
            double v[kMaxDegree + 1];
            int const jmin = eval_basis(D, b->points[d], v);
            if (d % 2 == 0) b->offset = jmin + d / 2 - d;
            else {
                int const mid = d / 2;
                b->offset = jmin + (v[mid] > v[mid + 1] ? mid : mid + 1) - d;
            }
        }
        SparseRows rows = assemble(*b);
        auto* priv = new BuilderPrivate();
        b->host_private = priv;
        priv->fwd.analyse(rows, D.periodic != 0);
        priv->fwd.make_tables(b->nchunk_req);
        priv->adj.analyse(transpose_rows(rows), D.periodic != 0);
        priv->adj.make_tables(b->nchunk_req);
        b->k = int(priv->fwd.k);
        b->m = int(priv->fwd.m);
        b->kl = int(priv->fwd.kl);
        b->ku = int(priv->fwd.ku);
        b->pivot = priv->fwd.pivot ? 1 : 0;
        b->structure = describe(priv->fwd);
        if (std::getenv("DDCB_DEBUG_PLAN")) std::fprintf(stderr, "ddcb plan: %s | adjoint %s\n", b->structure.c_str(), describe(priv->adj).c_str());
        // right-hand side map
        RhsMap& r = b->rhs;
        r.nbe_lo = b->nbe_lo;
        r.nbe_hi = b->nbe_hi;
        r.nbv_lo = b->nbv_lo;
        r.nbv_hi = b->nbv_hi;
        r.npoints = int(npts);
        r.offset = b->offset;
        r.size = int(b->basis.size());
        r.periodic = D.periodic;
        for (int i = 0; i < 8; ++i) {
            r.dxpow_lo[i] = ipow(b->dx, i + b->odd);
            r.dxpow_hi[i] = ipow(b->dx, i + b->odd);
        }
        // device tables (current device)
        int dev = 0;
        DDCB_CUDA_CHECK(cudaGetDevice(&dev));
        b->device = dev;
        upload_basis(b->basis, dev);
        std::vector<char> blob;
        std::vector<size_t> offs_f, offs_a;
        b->tables = upload_tables(priv->fwd, blob, offs_f);
        b->tables_t = upload_tables(priv->adj, blob, offs_a);
        DDCB_CUDA_CHECK(cudaMalloc(&b->d_block, blob.size()));
        DDCB_CUDA_CHECK(cudaMemcpy(b->d_block, blob.data(), blob.size(), cudaMemcpyHostToDevice));
        b->d_block_bytes = blob.size();
        bind_tables(b->tables, static_cast<char*>(b->d_block), offs_f.data());
        bind_tables(b->tables_t, static_cast<char*>(b->d_block), offs_a.data());
        return b;
    } catch (...) {
        destroy_builder(b);
        throw;
    }
}

void destroy_builder(Builder* b)
{
    if (!b) return;
    delete static_cast<BuilderPrivate*>(b->host_private);
    if (b->d_block) cudaFree(b->d_block);
    free_basis(b->basis);
    delete b;
}

// quadrature_coefficients (spline_builder.hpp:1103-1234): solve A^T q = integrals, un-rotate the
// periodic offset, split into Hermite / value parts and scale the Hermite parts by dx^k.
void builder_quadrature(Builder const& b, double* qlo, double* q, double* qhi)
{
    HostSolve const& h = static_cast<BuilderPrivate const*>(b.host_private)->fwd;
    std::vector<double> ints(b.basis.size());
    basis_integrals(b.basis, ints.data());
    // As the reference does, the right-hand side is integral_bsplines in basis order (entry j is
    // the integral of B-spline j), without the periodic column rotation.
    std::vector<double> rhs(b.n);
    for (long j = 0; j < b.n; ++j) rhs[j] = ints[j];
    h.solve_host(rhs.data(), true);
    long const nv = b.n - b.nbv_lo - b.nbv_hi;
    for (int i = 0; i < b.nbv_lo; ++i) qlo[i] = rhs[i] * ipow(b.dx, i + b.odd);
    for (long i = 0; i < nv; ++i) q[i] = rhs[b.nbv_lo + i];
    for (int i = 0; i < b.nbv_hi; ++i) qhi[i] = rhs[b.nbv_lo + nv + i] * ipow(b.dx, i + b.odd);
}

} // namespace ddcb
