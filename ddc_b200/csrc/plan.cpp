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

    void factor(bool pivoting = true)
    {
        ipiv.assign(m, 0);
        long ju = 0;
        for (long j = 0; j < m; ++j) {
            long const km = std::min(kl, m - 1 - j);
            long jp = 0;
            double amax = std::fabs(at(j, j));
            for (long t = 1; t <= km && pivoting; ++t)
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

    // || |L| |U| ||_inf of the factors (row i of |L||U| sums |l_ik| times the absolute row sum of
    // U's row k; the unit diagonal of L included): the quantity that bounds the backward error of
    // Gaussian elimination, |dA| <= gamma_3m |L||U| (Higham, Accuracy and Stability of Numerical
    // Algorithms, 2nd ed., Thm 9.3). With interchanges the multipliers are those of the row at
    // its elimination step, which is what partial pivoting bounds by 1.
    double growth() const
    {
        std::vector<double> r(size_t(m), 0.0);
        for (long k = 0; k < m; ++k)
            for (long t = 0; t <= kl + ku && k + t < m; ++t) r[size_t(k)] += std::fabs(at(k, k + t));
        double g = 0.0;
        for (long i = 0; i < m; ++i) {
            double s = r[size_t(i)];
            for (long t = 1; t <= kl && i - t >= 0; ++t) s += std::fabs(at(i, i - t)) * r[size_t(i - t)];
            g = std::max(g, s);
        }
        return g;
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
    long nchunk = 1, chunk_len = 0, chunk_split = 1, nscan = 0;
    long nscan_f = 0, nscan_b = 0; // scan steps run: later steps' transfers are below 2^-60
    std::vector<double> Lf, Uf, PhiF, PhiB;
    std::vector<int8_t> piv;
    long qg_lo = 0, qg_hi = 0;
    std::vector<double> qg_rows;
    std::vector<int> lam_row, lam_col;
    std::vector<double> lam_val;

    long chunk_begin(long c) const { return c * chunk_len + 2 * std::max(0L, c - chunk_split); }
    long chunk_end(long c) const { return (c == nchunk - 1) ? m : chunk_begin(c + 1); }

    // rows: the system in kernel order (the builder rotates the reference's boundary rows and
    // columns to the end); border: the number of trailing rows/cols solved through the Schur
    // complement (periodic systems: derived from the circular bandwidth instead).
    SparseRows sys; // the system in kernel order (kept for the FP64 residuals of the refinement)

    void analyse(SparseRows const& rows, bool periodic, long border)
    {
        sys = rows;
        n = long(rows.size());
        k = border;
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
        // Factorise without interchanges when that is as accurate as partial pivoting (the
        // interpolation block of B-spline collocation matrices is totally positive, for which
        // elimination without pivoting is stable: de Boor & Pinkus 1977); else pivot. Two checks,
        // both deterministic: (1) the growth || |L||U| ||_inf of the factors without interchanges
        // is at most 4x that of the pivoted factors, so the backward-error bound of Gaussian
        // elimination is within that factor of partial pivoting's; (2) on three fixed
        // pseudo-random right-hand sides (a fixed-seed LCG) the two solves agree to 1e-14.
        if (m > 0) {
            BandLU piv_lu = lu;
            piv_lu.factor(true);
            bool use_nopiv = true;
            try {
                lu.factor(false);
            } catch (Error const&) {
                use_nopiv = false;
            }
            if (use_nopiv && !(lu.growth() <= 4.0 * piv_lu.growth())) use_nopiv = false;
            if (use_nopiv) {
                std::vector<double> x1(m), x2(m);
                unsigned long long st = 0x9E3779B97F4A7C15ULL;
                for (int trial = 0; trial < 3 && use_nopiv; ++trial) {
                    for (long i = 0; i < m; ++i) {
                        st = st * 6364136223846793005ULL + 1442695040888963407ULL;
                        x1[i] = x2[i] = double(st >> 11) * (1.0 / 9007199254740992.0) - 0.5;
                    }
                    lu.solve(x1.data(), false);
                    piv_lu.solve(x2.data(), false);
                    double num = 0.0, den = 0.0;
                    for (long i = 0; i < m; ++i) {
                        num = std::max(num, std::fabs(x1[i] - x2[i]));
                        den = std::max(den, std::fabs(x2[i]));
                    }
                    if (!(num <= 1e-14 * den)) use_nopiv = false;
                }
            }
            if (!use_nopiv) lu = piv_lu;
        }
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
        // pad the bandwidths up to the cheapest band shape the kernels are compiled for
        // (build_kernels.cu dispatch)
        static long const shapes[][2] = {{1, 1}, {1, 2}, {2, 2}, {3, 3}, {1, 4}, {2, 4}, {4, 4}, {3, 6}, {1, 8}, {2, 8}, {4, 8}};
        long best = -1;
        for (long i = 0; i < long(sizeof(shapes) / sizeof(shapes[0])); ++i)
            if (shapes[i][0] >= std::max(kl, 1L) && shapes[i][1] >= std::max(ku, 1L)) {
                best = i;
                break;
            }
        if (best < 0)
            throw Error(DDCB_ERR_UNSUPPORTED, "band too wide for the device solver (kl=" + std::to_string(kl) + ", ku=" + std::to_string(ku) + ")");
        kl = shapes[best][0];
        ku = shapes[best][1];
        // lambda in compressed-row form (row i of the border: entries lam_ptr[i]..lam_ptr[i+1])
        lam_row.assign(1, 0);
        for (long i = 0; i < k; ++i) {
            for (long j = 0; j < m; ++j)
                if (lam[i * m + j] != 0.0) {
                    lam_col.push_back(int(j));
                    lam_val.push_back(lam[i * m + j]);
                }
            lam_row.push_back(int(lam_val.size()));
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
        // chunking: odd chunk lengths (conflict-free shared-memory rows), at least max(kl,ku)+1 rows.
        // Chunks have length L or L+2, so the longest sweep (the critical path) is at most two rows
        // above the average; when the remainder does not split that way the last chunk takes it.
        long const minlen = std::max<long>(std::max(kl, ku) + 1, 3);
        if (m == 0) {
            nchunk = 1;
            chunk_len = 0;
            chunk_split = 1;
        } else {
            long L = (m + nchunk_req - 1) / std::max<long>(nchunk_req, 1);
            L = std::max(L, minlen);
            if (L % 2 == 0) L += 1;
            nchunk = std::max<long>(1, m / L);
            chunk_split = nchunk;
            if (nchunk > 1) {
                long nc = nchunk, r = m - nc * L;
                if (r % 2) {
                    --nc;
                    r += L;
                }
                if (nc > 1 && r / 2 <= nc) {
                    nchunk = nc;
                    chunk_split = nc - r / 2;
                }
            }
            if (nchunk == 1) {
                L = m;
                chunk_split = 1;
            }
            chunk_len = L;
        }
        // transfer matrices of one chunk: Phi_c (forward, kl x kl), Psi_c (backward, ku x ku)
        std::vector<double> F(std::max<long>(nchunk * kl * kl, 1), 0.0), G(std::max<long>(nchunk * ku * ku, 1), 0.0);
        std::vector<double> w(std::max<long>(kl, 1)), z(std::max<long>(ku, 1));
        for (long c = 0; c < nchunk && m > 0; ++c) {
            long const a = chunk_begin(c), e = chunk_end(c);
            for (long s = 0; s < kl; ++s) {
                std::fill(w.begin(), w.end(), 0.0);
                w[s] = 1.0;
                fwd_steps(a, e, w.data());
                for (long r = 0; r < kl; ++r) F[(c * kl + r) * kl + s] = w[r];
            }
            for (long s = 0; s < ku; ++s) {
                std::fill(z.begin(), z.end(), 0.0);
                z[s] = 1.0;
                bwd_steps(a, e, z.data());
                for (long r = 0; r < ku; ++r) G[(c * ku + r) * ku + s] = z[r];
            }
        }
        // Products over runs of 2^k chunks for the log-depth carry scan (build_device.cuh):
        //   forward  P(k, c) = Phi_c Phi_{c-1} ... Phi_{c-2^k+1}
        //   backward Q(k, c) = Psi_c Psi_{c+1} ... Psi_{c+2^k-1}
        nscan = 0;
        while ((1L << nscan) < nchunk) ++nscan;
        PhiF.assign(std::max<long>(nscan * nchunk * kl * kl, 1), 0.0);
        PhiB.assign(std::max<long>(nscan * nchunk * ku * ku, 1), 0.0);
        auto matmul = [](double const* A, double const* B, double* C, long n) {
            for (long i = 0; i < n; ++i)
                for (long j = 0; j < n; ++j) {
                    double acc = 0.0;
                    for (long q = 0; q < n; ++q) acc += A[i * n + q] * B[q * n + j];
                    C[i * n + j] = acc;
                }
        };
        for (long k = 0; k < nscan; ++k) {
            long const half = (1L << k) / 2;
            for (long c = 0; c < nchunk; ++c) {
                double* Pf = &PhiF[(k * nchunk + c) * kl * kl];
                double* Pb = &PhiB[(k * nchunk + c) * ku * ku];
                if (k == 0) {
                    std::copy(&F[c * kl * kl], &F[(c + 1) * kl * kl], Pf);
                    std::copy(&G[c * ku * ku], &G[(c + 1) * ku * ku], Pb);
                    continue;
                }
                if (c - (1L << k) + 1 >= 0)
                    matmul(&PhiF[((k - 1) * nchunk + c) * kl * kl], &PhiF[((k - 1) * nchunk + c - half) * kl * kl], Pf, kl);
                if (c + (1L << k) - 1 <= nchunk - 1)
                    matmul(&PhiB[((k - 1) * nchunk + c) * ku * ku], &PhiB[((k - 1) * nchunk + c + half) * ku * ku], Pb, ku);
            }
        }
        // Step k of a scan adds P(k, c) times the true carry of chunk c -/+ 2^k; once every entry of
        // every P(k, .) is below 2^-60, that term and those of all later steps (products with
        // P(k, .) as a factor) are below FP64 rounding of the carries, so the scan stops there.
        auto steps_needed = [&](std::vector<double> const& Pm, long K) {
            for (long k = 0; k < nscan; ++k) {
                double mx = 0.0;
                for (long q = k * nchunk * K * K; q < (k + 1) * nchunk * K * K; ++q) mx = std::max(mx, std::fabs(Pm[q]));
                if (mx <= 0x1p-60) return k;
            }
            return nscan;
        };
        nscan_f = kl > 0 ? steps_needed(PhiF, kl) : 0;
        nscan_b = ku > 0 ? steps_needed(PhiB, ku) : 0;
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
    t.chunk_split = int(h.chunk_split);
    t.nscan = int(h.nscan);
    t.nscan_f = int(h.nscan_f);
    t.nscan_b = int(h.nscan_b);
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
    // The longest run of identical factor rows (the steady state a constant-coefficient band
    // reaches after a few rows) is stored once, so the tables of uniform meshes stay L1-resident.
    long const m = h.m, kl = h.kl, ku1 = h.ku + 1;
    auto same_row = [&](long i, long j) {
        return std::memcmp(&h.Lf[i * kl], &h.Lf[j * kl], sizeof(double) * kl) == 0
               && std::memcmp(&h.Uf[i * ku1], &h.Uf[j * ku1], sizeof(double) * ku1) == 0 && h.piv[i] == h.piv[j];
    };
    long best0 = m, best1 = m;
    for (long i = 0; i < m;) {
        long j = i + 1;
        while (j < m && same_row(i, j)) ++j;
        if (j - i > best1 - best0) {
            best0 = i;
            best1 = j;
        }
        i = j;
    }
    if (best1 - best0 < 8) best0 = best1 = m;
    t.cj0 = int(best0);
    t.cj1 = int(best1);
    t.cshift = best1 > best0 ? int(best1 - best0 - 1) : 0;
    // Without a steady run (non-uniform meshes) the chunks of a warp read different rows in every
    // sweep step; interleaving the rows by chunk makes those reads one contiguous segment.
    t.il = (best0 == m && h.nchunk > 1) ? 1 : 0;
    std::vector<double> Lc, Uc;
    std::vector<int8_t> pc;
    if (t.il) {
        long const NC = h.nchunk;
        long smax = 0;
        for (long c = 0; c < NC; ++c) smax = std::max(smax, h.chunk_end(c) - h.chunk_begin(c));
        Lc.assign(size_t(std::max<long>(smax * kl * NC, 1)), 0.0);
        Uc.assign(size_t(std::max<long>(smax * ku1 * NC, 1)), 0.0);
        pc.assign(size_t(std::max<long>(smax * NC, 1)), 0);
        for (long c = 0; c < NC; ++c) {
            long const a = h.chunk_begin(c), e = h.chunk_end(c);
            for (long j = a; j < e; ++j) {
                for (long q = 0; q < kl; ++q) Lc[size_t(factor_base(t, int(j), int(a), int(c), int(kl)) + q * NC)] = h.Lf[j * kl + q];
                for (long q = 0; q < ku1; ++q) Uc[size_t(factor_base(t, int(j), int(a), int(c), int(ku1)) + q * NC)] = h.Uf[j * ku1 + q];
                pc[size_t(piv_index(t, int(j), int(a), int(c)))] = h.piv[j];
            }
        }
    } else {
        for (long j = 0; j < m; ++j) {
            if (j > best0 && j < best1) continue;
            Lc.insert(Lc.end(), h.Lf.begin() + j * kl, h.Lf.begin() + (j + 1) * kl);
            Uc.insert(Uc.end(), h.Uf.begin() + j * ku1, h.Uf.begin() + (j + 1) * ku1);
            pc.push_back(h.piv[j]);
        }
    }
    // transfer products entry-major, [k][entry][chunk] (scan_index), so the chunks a warp scans
    // read one contiguous segment per entry
    auto entry_major = [&](std::vector<double> const& P, long K) {
        std::vector<double> o(P.size(), 0.0);
        long const NC = h.nchunk;
        for (long k = 0; k < h.nscan; ++k)
            for (long c = 0; c < NC; ++c)
                for (long e = 0; e < K * K; ++e) o[size_t(scan_index(t, int(k), int(e), int(c), int(K)))] = P[size_t((k * NC + c) * K * K + e)];
        return o;
    };
    std::vector<double> const PhiFc = entry_major(h.PhiF, kl), PhiBc = entry_major(h.PhiB, h.ku);
    push(Lc.data(), Lc.size() * 8);
    push(pc.data(), pc.size());
    push(Uc.data(), Uc.size() * 8);
    push(PhiFc.data(), PhiFc.size() * 8);
    push(PhiBc.data(), PhiBc.size() * 8);
    push(h.lam_row.data(), h.lam_row.size() * 4);
    push(h.lam_col.data(), h.lam_col.size() * 4);
    push(h.lam_val.data(), h.lam_val.size() * 8);
    push(h.Sinv.data(), h.Sinv.size() * 8);
    push(h.qg_rows.data(), h.qg_rows.size() * 8);
    // FP32 copies of the factor tables, in the order of SolveTables::F32
    auto push32 = [&](std::vector<double> const& v) {
        std::vector<float> f(v.begin(), v.end());
        push(f.data(), f.size() * 4);
    };
    push32(Lc);
    push32(Uc);
    push32(PhiFc);
    push32(PhiBc);
    push32(h.lam_val);
    push32(h.Sinv);
    push32(h.qg_rows);
    // the system matrix, CSR in kernel order
    std::vector<int> arow(1, 0), acol;
    std::vector<double> aval;
    for (auto const& r : h.sys) {
        for (auto const& [j, v] : r) {
            acol.push_back(int(j));
            aval.push_back(v);
        }
        arow.push_back(int(acol.size()));
    }
    push(arow.data(), arow.size() * 4);
    push(acol.data(), acol.size() * 4);
    push(aval.data(), aval.size() * 8);
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
    t.f32.Lf = reinterpret_cast<float const*>(base + offs[10]);
    t.f32.Uf = reinterpret_cast<float const*>(base + offs[11]);
    t.f32.PhiF = reinterpret_cast<float const*>(base + offs[12]);
    t.f32.PhiB = reinterpret_cast<float const*>(base + offs[13]);
    t.f32.lam_val = reinterpret_cast<float const*>(base + offs[14]);
    t.f32.Sinv = reinterpret_cast<float const*>(base + offs[15]);
    t.f32.Qg = reinterpret_cast<float const*>(base + offs[16]);
    t.a_row = reinterpret_cast<int const*>(base + offs[17]);
    t.a_col = reinterpret_cast<int const*>(base + offs[18]);
    t.a_val = reinterpret_cast<double const*>(base + offs[19]);
}

std::string describe(HostSolve const& h)
{
    return "border=" + std::to_string(h.k) + ",Q=BandLU(" + std::to_string(h.m) + ",kl=" + std::to_string(h.kl)
           + ",ku=" + std::to_string(h.ku) + (h.pivot ? ",pivoting" : "") + "),chunks=" + std::to_string(h.nchunk)
           + "x" + std::to_string(h.chunk_len) + ",scan=" + std::to_string(h.nscan_f) + "/" + std::to_string(h.nscan_b) + "of"
           + std::to_string(h.nscan);
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
    // A periodic basis of ncells <= degree wraps each B-spline onto itself (its support is longer
    // than the period), and the offset rule (spline_builder.hpp:619-658) reads interpolation point
    // number `degree`, which such a grid does not have.
    if (D.periodic && D.ncells <= D.degree)
        throw Error(DDCB_ERR_BAD_GRID, "a periodic basis of degree " + std::to_string(D.degree) + " needs more than "
                                           + std::to_string(D.degree) + " cells (got " + std::to_string(D.ncells) + ")");
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
    SparseRows ref_rows; // the assembled system in the reference's row / column order
};

// The system the reference solves on uniform bases. SplineBuilder::allocate_matrix passes
// pds = is_uniform() to the matrix maker (spline_builder.hpp:740-764), whose centre block -- rows
// and columns [top, n - bottom) of the 3x3 layout, or [0, n - max(kl, ku)) of the periodic 2x2
// layout, kl = ku = degree / 2 -- is then a symmetric band (splines_linear_problem_pds_band.cpp,
// pds_tridiag.cpp: entries (i, j) and (j, i) share one slot, entries beyond the band are dropped).
// build_matrix_system writes the rows in order (spline_builder.hpp:784-886), so each slot keeps
// its lower-triangle value when both were written. On the interpolation matrix of a uniform basis
// the two differ by round-off only, but that round-off moves the solution by up to cond(A) times
// it; solving the reference's symmetric block keeps the result within cond(A) eps of it.
static void symmetrize_like_reference(SparseRows& rows, Builder const& bl, long top, long bottom)
{
    BasisDesc const& D = bl.basis.desc;
    if (!D.uniform) return;
    long const n = bl.n, kd = D.degree / 2;
    long q0, q1;
    if (D.periodic) {
        long const bot = kd, tp = n - bot; // make_new_periodic_band_matrix: bottom = max(kl, ku)
        // its dense fallback keeps every entry as written
        if (bot * (n + tp) + (2 * kd + kd + 1) * tp >= n * n) return;
        q0 = 0;
        q1 = n - bot;
    } else {
        q0 = top;
        q1 = n - bottom;
    }
    for (long i = q0; i < q1; ++i)
        for (long j = i + 1; j < std::min(q1, i + kd + 1); ++j) {
            auto lo = rows[j].find(i);
            auto up = rows[i].find(j);
            // the later row (j) overwrites the slot when it wrote it
            double const v = lo != rows[j].end() ? lo->second : (up != rows[i].end() ? up->second : 0.0);
            if (v != 0.0) {
                rows[i][j] = v;
                rows[j][i] = v;
            }
        }
    // beyond the band, the centre block keeps nothing
    for (long i = q0; i < q1; ++i)
        for (auto it = rows[i].begin(); it != rows[i].end();) {
            long const j = it->first;
            if (j >= q0 && j < q1 && std::labs(j - i) > kd) it = rows[i].erase(it);
            else ++it;
        }
}

// An estimate of ||A^-1||_inf = ||A^-T||_1 by Higham's 1-norm estimator (N. J. Higham, ACM TOMS 14
// (1988) 381-396, after Hager 1984): a few solves with A^T and A on sign vectors. It bounds the
// forward error of a refined solution from its residual: |x - x*| <= ||A^-1|| |b - A x|.
static double inverse_norm_estimate(HostSolve const& h)
{
    long const n = h.n;
    if (n == 0) return 0.0;
    std::vector<double> x(n, 1.0 / double(n)), y(n), z(n);
    double est = 0.0;
    for (int it = 0; it < 5; ++it) {
        y = x;
        h.solve_host(y.data(), true); // y = A^-T x
        double e = 0.0;
        for (double v : y) e += std::fabs(v);
        if (it > 0 && e <= est) break;
        est = e;
        for (long i = 0; i < n; ++i) z[i] = y[i] >= 0.0 ? 1.0 : -1.0;
        h.solve_host(z.data(), false); // z = A^-1 sign(y)
        long j = 0;
        double zx = 0.0;
        for (long i = 0; i < n; ++i) {
            zx += z[i] * x[i];
            if (std::fabs(z[i]) > std::fabs(z[j])) j = i;
        }
        if (it > 0 && std::fabs(z[j]) <= zx) break;
        std::fill(x.begin(), x.end(), 0.0);
        x[j] = 1.0;
    }
    return est;
}

Builder* create_builder_host(Basis const& basis, double const* pts, long npts, int lo, int hi, ddcb_builder_options const* opts)
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
            if (opts->refine_rounds < 0 || opts->refine_rounds > 3)
                throw Error(DDCB_ERR_INVALID_ARGUMENT, "refine_rounds must be in 0..3 (0: the default, 2)");
            if (opts->refine_rounds > 0) b->refine_rounds = opts->refine_rounds;
            if (!(opts->refine_tolerance >= 0.0)) throw Error(DDCB_ERR_INVALID_ARGUMENT, "refine_tolerance must be >= 0");
            if (opts->refine_tolerance > 0.0) b->refine_tolerance = opts->refine_tolerance;
            if (opts->tile_lines > 0) b->tile_lines = opts->tile_lines;
            if (opts->chunks > 0) b->nchunk_req = opts->chunks;
        }
        if (b->tile_lines != 2 && b->tile_lines != 4 && b->tile_lines != 8 && b->tile_lines != 16)
            throw Error(DDCB_ERR_INVALID_ARGUMENT, "tile_lines must be 2, 4, 8 or 16");
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
        // Non-periodic systems: the reference's 3x3 block layout (splines_linear_problem_3x3_blocks.cpp,
        // block sizes of spline_builder.hpp:668-709) -- the first `top` rows/cols (Hermite rows,
        // Greville edge points) are rotated behind the band and, with the last `bottom`, form the
        // border; the band in between is the interpolation block.
        long top = 0, bottom = 0;
        if (!D.periodic) {
            auto block = [&](int bc, int nbc) -> long {
                if (D.uniform) return (bc == DDCB_GREVILLE) ? d - 1 : nbc;
                return (bc == DDCB_GREVILLE) ? d - 1 : nbc + 1;
            };
            top = block(lo, b->nbe_lo);
            bottom = block(hi, b->nbe_hi);
            if (top + bottom >= b->n) top = bottom = 0;
        }
        symmetrize_like_reference(rows, *b, top, bottom);
        b->rrot = int(top);
        b->crot = int(top);
        if (top) {
            long const nn = b->n;
            SparseRows rot(nn);
            for (long i = 0; i < nn; ++i)
                for (auto const& [j, v] : rows[(i + top) % nn]) rot[i][modulo(j - top, nn)] = v;
            rows.swap(rot);
        }
        auto* priv = new BuilderPrivate();
        b->host_private = priv;
        priv->ref_rows = assemble(*b);
        symmetrize_like_reference(priv->ref_rows, *b, top, bottom);
        priv->fwd.analyse(rows, D.periodic != 0, top + bottom);
        priv->fwd.make_tables(b->nchunk_req);
        priv->adj.analyse(transpose_rows(rows), D.periodic != 0, top + bottom);
        priv->adj.make_tables(b->nchunk_req);
        b->k = int(priv->fwd.k);
        b->m = int(priv->fwd.m);
        b->kl = int(priv->fwd.kl);
        b->ku = int(priv->fwd.ku);
        b->pivot = priv->fwd.pivot ? 1 : 0;
        b->structure = describe(priv->fwd);
        {
            // cond_inf(A) = ||A||_inf ||A^-1||_inf, the factor of the refinement's error bound
            double anorm = 0.0;
            for (auto const& row : priv->ref_rows) {
                double s = 0.0;
                for (auto const& [j, v] : row) s += std::fabs(v);
                anorm = std::max(anorm, s);
            }
            b->cond_est = anorm * inverse_norm_estimate(priv->fwd);
        }
        if (std::getenv("DDCB_DEBUG_PLAN")) {
            std::fprintf(stderr, "ddcb plan: %s | adjoint %s\n", b->structure.c_str(), describe(priv->adj).c_str());
            std::fprintf(stderr, "  swaps at:");
            for (long j = 0; j < priv->fwd.m; ++j)
                if (priv->fwd.lu.ipiv[j] != j) std::fprintf(stderr, " %ld->%d", j, priv->fwd.lu.ipiv[j]);
            std::fprintf(stderr, "\n  lu.kl=%ld lu.ku=%ld\n", priv->fwd.lu.kl, priv->fwd.lu.ku);
        }
        // right-hand side map
        RhsMap& r = b->rhs;
        r.nbe_lo = b->nbe_lo;
        r.nbe_hi = b->nbe_hi;
        r.nbv_lo = b->nbv_lo;
        r.nbv_hi = b->nbv_hi;
        r.npoints = int(npts);
        r.offset = b->offset;
        r.lrot = b->rrot;
        r.srot = (b->offset + b->crot) % int(b->n);
        r.size = int(b->basis.size());
        r.periodic = D.periodic;
        for (int i = 0; i < 8; ++i) {
            r.dxpow_lo[i] = ipow(b->dx, i + b->odd);
            r.dxpow_hi[i] = ipow(b->dx, i + b->odd);
        }
        return b;
    } catch (...) {
        destroy_builder(b);
        throw;
    }
}

void upload_builder(Builder* b)
{
    auto* priv = static_cast<BuilderPrivate*>(b->host_private);
    int dev = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    b->device = dev;
    upload_basis(b->basis, dev);
    std::vector<char> blob;
    std::vector<size_t> offs_f, offs_a;
    b->tables = upload_tables(priv->fwd, blob, offs_f);
    b->tables_t = upload_tables(priv->adj, blob, offs_a);
    // the quadrature weights and their scratch (2 n doubles) follow the tables, then the
    // interpolation points (the advection step's feet start from them)
    size_t const qoff = (blob.size() + 255) & ~size_t(255);
    size_t const nw = size_t(b->basis.size()) + b->points.size() + size_t(b->nbv_lo + b->nbv_hi);
    size_t const poff = qoff + sizeof(double) * (2 * size_t(b->n) + nw);
    size_t const soff = poff + sizeof(double) * b->points.size();
    blob.resize(soff + 8, 0);
    std::memcpy(blob.data() + poff, b->points.data(), sizeof(double) * b->points.size());
    DDCB_CUDA_CHECK(cudaMalloc(&b->d_block, blob.size()));
    DDCB_CUDA_CHECK(cudaMemcpy(b->d_block, blob.data(), blob.size(), cudaMemcpyHostToDevice));
    b->d_block_bytes = blob.size();
    bind_tables(b->tables, static_cast<char*>(b->d_block), offs_f.data());
    bind_tables(b->tables_t, static_cast<char*>(b->d_block), offs_a.data());
    b->d_quad_scratch = reinterpret_cast<double*>(static_cast<char*>(b->d_block) + qoff);
    b->d_quad = b->d_quad_scratch + b->n;
    b->d_iweights = b->d_quad + b->n + b->basis.size();
    b->d_points = reinterpret_cast<double*>(static_cast<char*>(b->d_block) + poff);
    b->d_status = reinterpret_cast<unsigned*>(static_cast<char*>(b->d_block) + soff);
    b->tables.cond_est = b->tables_t.cond_est = b->cond_est;
    b->tables.refine_tol = b->tables_t.refine_tol = b->refine_tolerance;
    b->tables.status = b->tables_t.status = b->d_status;
}

Builder* create_builder(Basis const& basis, double const* pts, long npts, int lo, int hi, ddcb_builder_options const* opts)
{
    Builder* b = create_builder_host(basis, pts, npts, lo, hi, opts);
    try {
        upload_builder(b);
    } catch (...) {
        destroy_builder(b);
        throw;
    }
    return b;
}

// Runs, on the host, exactly the steps the device solve performs (chunked sweeps with the carry
// scan, border correction) on one right-hand side and returns its max-norm distance to the direct
// host solve, relative to the solution's max norm. Used by the host-side tests of the plan.
static void emulate_tile_solve(HostSolve const& h, std::vector<double>& T);

double emulate_device_solve(Builder const& b, double const* rhs, bool transpose)
{
    HostSolve const& h = transpose ? static_cast<BuilderPrivate const*>(b.host_private)->adj
                                   : static_cast<BuilderPrivate const*>(b.host_private)->fwd;
    long const n = h.n;
    std::vector<double> T(rhs, rhs + n), ref(rhs, rhs + n);
    h.solve_host(ref.data(), false); // h is already the transposed system when transpose is set
    emulate_tile_solve(h, T);
    double num = 0.0, den = 0.0;
    for (long i = 0; i < n; ++i) {
        num = std::max(num, std::fabs(T[i] - ref[i]));
        den = std::max(den, std::fabs(ref[i]));
    }
    return num / std::max(den, 1e-300);
}

// Host replay of one device build of a single line: right-hand side gather with the row
// rotation and Hermite scaling, tile solve, store with the column rotation and periodic copies.
// Returns the max-norm distance (relative) to a dense Gaussian elimination of the system in the
// reference's order followed by the reference's placement of the solution
// (spline_builder.hpp:981-1100).
double emulate_build(Builder const& b, double const* vals, double const* dlo, double const* dhi)
{
    auto const* priv = static_cast<BuilderPrivate const*>(b.host_private);
    HostSolve const& h = priv->fwd;
    RhsMap const& R = b.rhs;
    long const n = b.n;
    std::vector<double> T(n, 0.0);
    bool const all_vals = R.periodic != 0;
    long const v0 = all_vals ? 0 : R.nbe_lo, v1 = all_vals ? n : R.nbe_lo + R.npoints;
    for (long r = 0; r < n; ++r) {
        long const sr = (r + R.lrot) % n;
        if (sr >= v0 && sr < v1) T[r] = vals[sr - v0];
        else if (sr < R.nbe_lo) T[r] = sr < R.nbv_lo ? dlo[sr] * R.dxpow_lo[sr] : 0.0;
        else {
            long const i = sr - (n - R.nbe_hi);
            T[r] = i < R.nbv_hi ? dhi[i] * R.dxpow_hi[i] : 0.0;
        }
    }
    emulate_tile_solve(h, T);
    std::vector<double> out(R.size);
    for (long o = 0; o < R.size; ++o) {
        long src = (o % n) - R.srot;
        src = ((src % n) + n) % n;
        out[o] = T[src];
    }
    // reference: dense system in reference order, rhs = [dlo*dx^k | vals | dhi*dx^k]
    std::vector<double> A(n * n, 0.0), x(n, 0.0);
    for (long i = 0; i < n; ++i)
        for (auto const& [j, v] : priv->ref_rows[i]) A[i * n + j] = v;
    for (long i = 0; i < n; ++i) {
        if (all_vals) x[i] = vals[i];
        else if (i < R.nbe_lo) x[i] = i < R.nbv_lo ? dlo[i] * R.dxpow_lo[i] : 0.0;
        else if (i < R.nbe_lo + R.npoints) x[i] = vals[i - R.nbe_lo];
        else {
            long const q = i - (n - R.nbe_hi);
            x[i] = q < R.nbv_hi ? dhi[q] * R.dxpow_hi[q] : 0.0;
        }
    }
    for (long c = 0; c < n; ++c) { // Gaussian elimination with partial pivoting
        long p = c;
        for (long i = c + 1; i < n; ++i)
            if (std::fabs(A[i * n + c]) > std::fabs(A[p * n + c])) p = i;
        if (p != c) {
            for (long j = 0; j < n; ++j) std::swap(A[c * n + j], A[p * n + j]);
            std::swap(x[c], x[p]);
        }
        for (long i = c + 1; i < n; ++i) {
            double const f = A[i * n + c] / A[c * n + c];
            if (f == 0.0) continue;
            for (long j = c; j < n; ++j) A[i * n + j] -= f * A[c * n + j];
            x[i] -= f * x[c];
        }
    }
    for (long c = n - 1; c >= 0; --c) {
        double s = x[c];
        for (long j = c + 1; j < n; ++j) s -= A[c * n + j] * x[j];
        x[c] = s / A[c * n + c];
    }
    // column j of the reference system is B-spline (j + offset) mod n; rows n.. repeat rows 0..
    std::vector<double> ref(R.size);
    for (long j = 0; j < n; ++j) ref[(j + R.offset) % n] = x[j];
    for (long o = n; o < R.size; ++o) ref[o] = ref[o - n];
    double num = 0.0, den = 0.0;
    for (long o = 0; o < R.size; ++o) {
        num = std::max(num, std::fabs(out[o] - ref[o]));
        den = std::max(den, std::fabs(ref[o]));
    }
    return num / std::max(den, 1e-300);
}

static void emulate_tile_solve(HostSolve const& h, std::vector<double>& T)
{
    long const m = h.m, k = h.k, KL = h.kl, KU = h.ku, NC = h.nchunk;
    // the factor and transfer tables as the kernels receive them, read with the kernels' indexing
    std::vector<char> blob;
    std::vector<size_t> offs;
    SolveTables tb = upload_tables(h, blob, offs);
    bind_tables(tb, blob.data(), offs.data());
    long const qs = factor_stride(tb);
    auto Lf_at = [&](long j, long a, long c, long q) { return tb.Lf[factor_base(tb, int(j), int(a), int(c), int(KL)) + q * qs]; };
    auto Uf_at = [&](long j, long a, long c, long q) { return tb.Uf[factor_base(tb, int(j), int(a), int(c), int(KU + 1)) + q * qs]; };
    auto piv_at = [&](long j, long a, long c) { return long(tb.piv[piv_index(tb, int(j), int(a), int(c))]); };
    std::vector<double> carry(NC * std::max(KL, KU), 0.0), halo(NC * KL, 0.0);
    auto scan = [&](double const* P, long K, bool fwd) {
        std::vector<double> y(carry);
        for (long s = 0; s < (fwd ? tb.nscan_f : tb.nscan_b); ++s) {
            std::vector<double> next(y);
            for (long c = 0; c < NC; ++c) {
                long const nb = fwd ? c - (1L << s) : c + (1L << s);
                if (nb < 0 || nb >= NC) continue;
                for (long r = 0; r < K; ++r) {
                    double acc = y[c * K + r];
                    for (long q = 0; q < K; ++q) acc += P[scan_index(tb, int(s), int(r * K + q), int(c), int(K))] * y[nb * K + q];
                    next[c * K + r] = acc;
                }
            }
            y = next;
        }
        carry = y;
    };
    if (m > 0) {
        // forward, phase A
        carry.assign(NC * KL, 0.0);
        for (long c = 0; c < NC; ++c) {
            long const a = h.chunk_begin(c), e = h.chunk_end(c);
            std::vector<double> w(KL + 1, 0.0);
            for (long q = 0; q < KL; ++q) w[q] = (a + q < m) ? T[a + q] : 0.0;
            for (long j = a; j < e; ++j) {
                w[KL] = (j + KL < m) ? T[j + KL] : 0.0;
                long const p = piv_at(j, a, c);
                if (p) std::swap(w[0], w[p]);
                double const y = w[0];
                for (long q = 1; q <= KL; ++q) w[q] -= Lf_at(j, a, c, q - 1) * y;
                for (long q = 0; q < KL; ++q) w[q] = w[q + 1];
            }
            for (long q = 0; q < KL; ++q) {
                double const orig = (e + q < m) ? T[e + q] : 0.0;
                carry[c * KL + q] = w[q] - orig;
                halo[c * KL + q] = orig;
            }
        }
        scan(tb.PhiF, KL, true);
        std::vector<double> Tn(T);
        for (long c = 0; c < NC; ++c) {
            long const a = h.chunk_begin(c), e = h.chunk_end(c);
            std::vector<double> w(KL + 1, 0.0);
            for (long q = 0; q < KL; ++q) w[q] = (a + q < m) ? T[a + q] + (c > 0 ? carry[(c - 1) * KL + q] : 0.0) : 0.0;
            for (long j = a; j < e; ++j) {
                long const rr = j + KL;
                w[KL] = rr < e ? T[rr] : (rr < m ? halo[c * KL + rr - e] : 0.0);
                long const p = piv_at(j, a, c);
                if (p) std::swap(w[0], w[p]);
                double const y = w[0];
                Tn[j] = y;
                for (long q = 1; q <= KL; ++q) w[q] -= Lf_at(j, a, c, q - 1) * y;
                for (long q = 0; q < KL; ++q) w[q] = w[q + 1];
            }
        }
        T = Tn;
        // backward
        carry.assign(NC * KU, 0.0);
        for (long c = 0; c < NC; ++c) {
            long const a = h.chunk_begin(c), e = h.chunk_end(c);
            std::vector<double> z(KU, 0.0);
            for (long j = e - 1; j >= a; --j) {
                double s = T[j];
                for (long q = 1; q <= KU; ++q) s -= Uf_at(j, a, c, q) * z[q - 1];
                double const x = s * Uf_at(j, a, c, 0);
                for (long q = KU - 1; q >= 1; --q) z[q] = z[q - 1];
                z[0] = x;
            }
            for (long q = 0; q < KU; ++q) carry[c * KU + q] = z[q];
        }
        scan(tb.PhiB, KU, false);
        for (long c = 0; c < NC; ++c) {
            long const a = h.chunk_begin(c), e = h.chunk_end(c);
            std::vector<double> z(KU, 0.0);
            for (long q = 0; q < KU; ++q) z[q] = (c + 1 < NC) ? carry[(c + 1) * KU + q] : 0.0;
            for (long j = e - 1; j >= a; --j) {
                double s = T[j];
                for (long q = 1; q <= KU; ++q) s -= Uf_at(j, a, c, q) * z[q - 1];
                double const x = s * Uf_at(j, a, c, 0);
                Tn[j] = x;
                for (long q = KU - 1; q >= 1; --q) z[q] = z[q - 1];
                z[0] = x;
            }
        }
        T = Tn;
    }
    if (k > 0) {
        std::vector<double> bt(k);
        for (long r = 0; r < k; ++r) bt[r] = T[m + r];
        for (long r = 0; r < k; ++r)
            for (int q = h.lam_row[r]; q < h.lam_row[r + 1]; ++q) bt[r] -= h.lam_val[q] * T[h.lam_col[q]];
        for (long r = 0; r < k; ++r) {
            double s = 0.0;
            for (long q = 0; q < k; ++q) s += h.Sinv[r * k + q] * bt[q];
            T[m + r] = s;
        }
        long const nq = h.qg_lo + h.qg_hi;
        for (long q = 0; q < nq; ++q) {
            long const i = q < h.qg_lo ? q : m - h.qg_hi + (q - h.qg_lo);
            for (long r = 0; r < k; ++r) T[i] -= h.qg_rows[q * k + r] * T[m + r];
        }
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

} // namespace ddcb
