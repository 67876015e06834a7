// Optimized breakup of a periodic pair function (Natoli & Ceperley 1995).
// See alea_breakup.h for the method; this file holds the quadrature, the
// Hermite shape functions, the χ² fit and the transforms of the two pair
// functions the walker path splits (Coulomb and the Padé Jastrow's rational
// u(r) − u(∞)).
#include "alea_breakup.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <stdexcept>
#include <thread>

namespace alea_breakup {
namespace {

constexpr double kPi = 3.14159265358979323846;

// ───────────────────────── quadrature ─────────────────────────────────

// n-point Gauss-Legendre rule on [-1, 1]: nodes by Newton's method on P_n
// from the Bonnet recurrence, started at Tricomi's approximation
// cos(π(i − 1/4)/(n + 1/2)); weights 2 / ((1 − x²) P_n'(x)²).
struct Rule {
    std::vector<double> x, w;
    explicit Rule(int n) {
        for (int i = 1; i <= n; ++i) {
            double z = std::cos(kPi * (i - 0.25) / (n + 0.5)), dp = 0.0;
            for (int it = 0; it < 100; ++it) {
                double p0 = 1.0, p1 = z;
                for (int m = 2; m <= n; ++m) {
                    const double p2 = ((2.0 * m - 1.0) * z * p1 - (m - 1.0) * p0) / m;
                    p0 = p1;
                    p1 = p2;
                }
                dp = n * (z * p1 - p0) / (z * z - 1.0);
                const double step = p1 / dp;
                z -= step;
                if (std::abs(step) < 1e-16) break;
            }
            x.push_back(z);
            w.push_back(2.0 / ((1.0 - z * z) * dp * dp));
        }
    }
};

const Rule& rule16() {
    static const Rule r(16);
    return r;
}

// ∫_a^b g over `pieces` equal sub-intervals with the 16-point rule.
template <class G>
double integrate(G&& g, double a, double b, int pieces) {
    const Rule& q = rule16();
    const double h = (b - a) / pieces;
    double total = 0.0;
    for (int p = 0; p < pieces; ++p) {
        const double mid = a + (p + 0.5) * h, half = 0.5 * h;
        double s = 0.0;
        for (size_t i = 0; i < q.x.size(); ++i) s += q.w[i] * g(mid + half * q.x[i]);
        total += half * s;
    }
    return total;
}

// Sub-intervals for ∫_a^b of an integrand oscillating with phase k r and
// varying on the length `scale` (0: no such limit): at most 4 radians of
// phase and half a scale per piece.
int pieces_for(double a, double b, double k, double scale) {
    double n = 1.0 + std::floor(k * (b - a) / 4.0);
    if (scale > 0.0) n = std::max(n, std::ceil(2.0 * (b - a) / scale));
    return static_cast<int>(std::min(n, 1e6));
}

// ───────────────────────── radial kernel ──────────────────────────────

// J0 of the 2-D transform: the library function below x = 25; above, the
// Hankel expansion J0 = √(2/πx) (P cos χ − Q sin χ), χ = x − π/4, with
// P = t0 − t2 + t4 − …, Q = −(t1 − t3 + …) and
// t_m = t_{m−1} (2m − 1)² / (8 m x) (Abramowitz & Stegun 9.2.5, 9.2.9-10 at
// ν = 0), summed until the terms fall below 1e-17 (they shrink while
// m < 2x, so at x ≥ 25 the truncation error is far below rounding).
double bessel_j0(double x) {
    if (x < 25.0) return std::cyl_bessel_j(0.0, x);
    double p = 1.0, q = 0.0, t = 1.0;
    for (int m = 1; m < 200; ++m) {
        const double next = t * (2.0 * m - 1.0) * (2.0 * m - 1.0) / (8.0 * m * x);
        if (next > t) break;
        t = next;
        switch (m & 3) {
            case 1: q -= t; break;
            case 2: p -= t; break;
            case 3: q += t; break;
            default: p += t; break;
        }
        if (t < 1e-17) break;
    }
    const double c = std::cos(x), s = std::sin(x);
    const double cchi = (c + s) * 0.70710678118654752440, schi = (s - c) * 0.70710678118654752440;
    return std::sqrt(2.0 / (kPi * x)) * (p * cchi - q * schi);
}

// ∫ f(|r|) e^{−ik·r} dᵈr = ∫_0^∞ kernel(d, k, r) f(r) dr.
double kernel(int dim, double k, double r) {
    if (dim == 2) return 2.0 * kPi * r * bessel_j0(k * r);
    return k > 0.0 ? 4.0 * kPi * r * std::sin(k * r) / k : 4.0 * kPi * r * r;
}

// ───────────────────────── Wynn's ε algorithm ─────────────────────────

// Accelerates a sequence of partial sums (Wynn, MTAC 10, 91 (1956)).  Each
// push adds S_n and returns the highest even-order estimate of the limit.
class Epsilon {
public:
    double push(double s) {
        std::vector<double> cur(diag_.size() + 1);
        cur[0] = s;
        double best = s;
        for (size_t m = 0; m < diag_.size(); ++m) {
            const double diff = cur[m] - diag_[m];
            if (diff == 0.0) {
                cur.resize(m + 1);
                break;
            }
            cur[m + 1] = (m >= 1 ? diag_[m - 1] : 0.0) + 1.0 / diff;
            if ((m + 1) % 2 == 0) best = cur[m + 1];
        }
        diag_ = std::move(cur);
        return best;
    }

private:
    std::vector<double> diag_;   // ε_m of the previous anti-diagonal
};

// ───────────────────────── pair functions ─────────────────────────────

class Coulomb final : public PairFunction {
public:
    explicit Coulomb(double inner_floor) : floor_(inner_floor) {}
    void eval(double r, double& f, double& df, double& d2f) const override {
        f = 1.0 / r;
        df = -f * f;
        d2f = -2.0 * df * f;
    }
    double inside(int dim, double rc, double k) const override {
        const double r0 = floor_ * rc;
        if (dim == 3)
            return k > 0.0 ? 4.0 * kPi * (std::cos(k * r0) - std::cos(k * rc)) / (k * k)
                           : 2.0 * kPi * (rc * rc - r0 * r0);
        if (k == 0.0) return 2.0 * kPi * (rc - r0);
        return 2.0 * kPi * integrate([&](double r) { return bessel_j0(k * r); }, r0, rc,
                                     pieces_for(r0, rc, k, 0.0));
    }
    double outside(int dim, double rc, double k) const override {
        if (dim == 3) return 4.0 * kPi / (k * k) - inside(dim, rc, k);
        return 2.0 * kPi / k - inside(dim, rc, k);
    }

private:
    double floor_;
};

class Rational final : public PairFunction {
public:
    Rational(std::vector<double> num, std::vector<double> den) {
        while (!num.empty() && num.back() == 0.0) num.pop_back();
        while (!den.empty() && den.back() == 0.0) den.pop_back();
        if (num.size() > den.size())
            throw std::invalid_argument("pair function: a numerator of higher degree than the denominator has no limit");
        p_.assign(1, 0.0);
        p_.insert(p_.end(), num.begin(), num.end());
        q_.assign(1, 1.0);
        q_.insert(q_.end(), den.begin(), den.end());
        limit_ = (!num.empty() && num.size() == den.size()) ? num.back() / den.back() : 0.0;
        // Fujiwara's bound on the roots of Q's reversal: every root z of Q has
        // |z| ≥ 1 / (2 max_i |q_i|^{1/i}).
        double m = 0.0;
        for (size_t i = 1; i < q_.size(); ++i) m = std::max(m, std::pow(std::abs(q_[i]), 1.0 / i));
        scale_ = m > 0.0 ? 0.5 / m : 0.0;
        for (int i = 0; i <= 2000; ++i) {
            const double r = 1e-6 * std::pow(10.0, 14.0 * i / 2000.0);
            double q = 0.0;
            for (size_t j = q_.size(); j-- > 0;) q = q * r + q_[j];
            if (!(q > 0.0)) throw std::invalid_argument("pair function: the denominator vanishes at some r > 0");
        }
    }
    double limit() const { return limit_; }

    void eval(double r, double& f, double& df, double& d2f) const override {
        double P[3], Q[3];
        horner(p_, r, P);
        horner(q_, r, Q);
        const double u = P[0] / Q[0];
        const double du = (P[1] - u * Q[1]) / Q[0];
        f = u - limit_;
        df = du;
        d2f = (P[2] - 2.0 * du * Q[1] - u * Q[2]) / Q[0];
    }

    // ∫_{r_c}^∞ between successive zeros of the kernel's oscillating factor
    // (2-D: J0(kr), whose zeros approach kr = (m + 3/4)π; 3-D: sin(kr) = 0 at
    // kr = mπ): the pieces alternate in sign with slowly varying size, and
    // the ε algorithm sums them to rounding in a few dozen terms.
    double outside(int dim, double rc, double k) const override {
        const double shift = dim == 2 ? 0.75 : 0.0;
        auto g = [&](double r) { return kernel(dim, k, r) * value(r); };
        double m = std::floor(k * rc / kPi - shift) + 1.0;
        double lo = rc, partial = 0.0, biggest = 0.0, last = 0.0;
        Epsilon eps;
        int steady = 0;
        for (int term = 0; term < 400; ++term, m += 1.0) {
            const double hi = (m + shift) * kPi / k;
            partial += integrate(g, lo, hi, pieces_for(lo, hi, k, scale_));
            lo = hi;
            biggest = std::max(biggest, std::abs(partial));
            const double est = eps.push(partial);
            if (term >= 6 && std::abs(est - last) <= 1e-15 * biggest) {
                if (++steady == 3) return est;
            } else {
                steady = 0;
            }
            last = est;
        }
        return last;
    }

protected:
    double scale() const override { return scale_; }

private:
    // c(r), c'(r), c''(r) of Σ c_i rⁱ
    static void horner(const std::vector<double>& c, double r, double out[3]) {
        double v = 0.0, d1 = 0.0, d2 = 0.0;
        for (size_t i = c.size(); i-- > 0;) {
            d2 = d2 * r + d1;
            d1 = d1 * r + v;
            v = v * r + c[i];
        }
        out[0] = v;
        out[1] = d1;
        out[2] = 2.0 * d2;
    }
    std::vector<double> p_, q_;
    double limit_ = 0.0, scale_ = 0.0;
};

// ───────────────────────── Hermite pieces ─────────────────────────────

// Quintic Hermite shape functions on t ∈ [0, 1]: H0 carries the value, H1
// the slope, H2 the curvature at t = 0, and all three with their first two
// derivatives vanish at t = 1 (H0 = (1−t)³(1+3t+6t²), H1 = t(1−t)³(1+3t),
// H2 = t²(1−t)³/2).
inline void hermite(double t, double h[3]) {
    const double u = 1.0 - t, u3 = u * u * u;
    h[0] = u3 * (1.0 + t * (3.0 + 6.0 * t));
    h[1] = t * u3 * (1.0 + 3.0 * t);
    h[2] = 0.5 * t * t * u3;
}

// Transforms of the 3·n_knots knot functions at k: segment by segment, the
// six functions living on a segment (three of its left knot, three of its
// right, the latter by reflection t → 1 − t with the slope's sign flipped)
// share the quadrature nodes.
void knot_transforms(int dim, int n_knots, double delta, double k, double* out) {
    std::fill(out, out + 3 * n_knots, 0.0);
    const Rule& q = rule16();
    const double scale[3] = {1.0, delta, delta * delta};
    for (int s = 0; s + 1 < n_knots; ++s) {
        const double a = s * delta, b = a + delta;
        const int pieces = pieces_for(a, b, k, 0.0);
        const double h = delta / pieces;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int p = 0; p < pieces; ++p) {
            const double mid = a + (p + 0.5) * h, half = 0.5 * h;
            for (size_t i = 0; i < q.x.size(); ++i) {
                const double r = mid + half * q.x[i];
                const double w = q.w[i] * half * kernel(dim, k, r);
                const double t = (r - a) / delta;
                double hl[3], hr[3];
                hermite(t, hl);
                hermite(1.0 - t, hr);
                for (int m = 0; m < 3; ++m) {
                    acc[m] += w * hl[m];
                    acc[3 + m] += w * hr[m];
                }
            }
        }
        for (int m = 0; m < 3; ++m) {
            out[3 * s + m] += acc[m] * scale[m];
            out[3 * (s + 1) + m] += (m == 1 ? -acc[3 + m] : acc[3 + m]) * scale[m];
        }
    }
}

// body(i) for i < n, strided over the host's hardware threads.
template <class F>
void strided_threads(size_t n, F&& body) {
    const size_t nt = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), (n + 3) / 4);
    if (nt <= 1) {
        for (size_t i = 0; i < n; ++i) body(i);
        return;
    }
    std::vector<std::thread> team;
    for (size_t t = 0; t < nt; ++t)
        team.emplace_back([&, t] {
            for (size_t i = t; i < n; i += nt) body(i);
        });
    for (auto& th : team) th.join();
}

// Integer bound per axis of the box holding every lattice vector with
// |k| ≤ kmax: n_i = k · a_i / 2π.
void index_bounds(const Lattice& lat, double kmax, int nb[3]) {
    for (int i = 0; i < 3; ++i) {
        double a2 = 0.0;
        for (int d = 0; d < lat.dim; ++d) a2 += lat.a[i * lat.dim + d] * lat.a[i * lat.dim + d];
        nb[i] = i < lat.dim ? static_cast<int>(kmax * std::sqrt(a2) / (2.0 * kPi)) + 1 : 0;
    }
}

// k = Σ n_i b_i and its length (hypot in 2-D, so that vectors on a shell
// boundary fall on the same side in every build).
double kvector(const Lattice& lat, const int n[3], double k[3]) {
    for (int d = 0; d < 3; ++d) k[d] = 0.0;
    for (int i = 0; i < lat.dim; ++i)
        for (int d = 0; d < lat.dim; ++d) k[d] += n[i] * lat.b[i * lat.dim + d];
    if (lat.dim == 2) return std::hypot(k[0], k[1]);
    return std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
}

}  // namespace

double PairFunction::inside(int dim, double rc, double k) const {
    return integrate([&](double r) { return kernel(dim, k, r) * value(r); }, 0.0, rc,
                     std::max(2, pieces_for(0.0, rc, k, scale())));
}

std::unique_ptr<PairFunction> coulomb(double inner_floor) { return std::make_unique<Coulomb>(inner_floor); }

std::unique_ptr<PairFunction> rational(std::vector<double> num, std::vector<double> den, double* limit) {
    auto f = std::make_unique<Rational>(std::move(num), std::move(den));
    if (limit) *limit = f->limit();
    return f;
}

Result optimize(const Lattice& lat, double rc, const PairFunction& f, const Options& opt) {
    const int dim = lat.dim;
    if ((dim != 2 && dim != 3) || !(rc > 0.0) || !(lat.volume > 0.0) || opt.n_knots < 2 || opt.n_continuum < 1)
        throw std::invalid_argument("breakup: bad lattice, cutoff or options");
    double b_min = 0.0;
    for (int i = 0; i < dim; ++i) {
        double b2 = 0.0;
        for (int d = 0; d < dim; ++d) b2 += lat.b[i * dim + d] * lat.b[i * dim + d];
        b_min = i == 0 ? std::sqrt(b2) : std::min(b_min, std::sqrt(b2));
    }
    Result R;
    R.n_knots = opt.n_knots;
    R.rc = rc;
    R.delta = rc / (opt.n_knots - 1);
    R.k_cut = opt.k_cut > 0.0 ? opt.k_cut : 8.0 * b_min;
    const double k_cont = opt.k_continuum > 0.0 ? opt.k_continuum : 60.0 * kPi / rc;
    const double k_max = opt.k_max > 0.0 ? opt.k_max : 6000.0 / rc;
    if (!(R.k_cut < k_cont && k_cont < k_max))
        throw std::invalid_argument("breakup: need k_cut < k_continuum < k_max");

    // χ² rows: each distinct |k| of the lattice in (k_cut, k_continuum] with
    // its number of vectors, then the continuum, ∫ dk of the density of
    // vectors (V/2π) k (2-D) or (V/2π²) k² (3-D), by the midpoint rule in
    // ln k.
    std::vector<double> row_k, row_w;
    size_t n_shell_rows = 0;
    {
        int nb[3];
        index_bounds(lat, k_cont, nb);
        std::vector<double> ks;
        int n[3];
        for (n[0] = -nb[0]; n[0] <= nb[0]; ++n[0])
            for (n[1] = -nb[1]; n[1] <= nb[1]; ++n[1])
                for (n[2] = -nb[2]; n[2] <= nb[2]; ++n[2]) {
                    if (n[0] == 0 && n[1] == 0 && n[2] == 0) continue;
                    double k[3];
                    const double kk = kvector(lat, n, k);
                    if (kk > R.k_cut && kk <= k_cont) ks.push_back(kk);
                }
        std::sort(ks.begin(), ks.end());
        for (double kk : ks) {
            if (!row_k.empty() && kk - row_k.back() < 1e-12 * kk) {
                row_w.back() += 1.0;
            } else {
                row_k.push_back(kk);
                row_w.push_back(1.0);
            }
        }
        n_shell_rows = row_k.size();
        const double l0 = std::log(k_cont), dl = (std::log(k_max) - l0) / opt.n_continuum;
        for (int i = 0; i < opt.n_continuum; ++i) {
            const double kk = std::exp(l0 + (i + 0.5) * dl);
            const double density = dim == 2 ? lat.volume * kk / (2.0 * kPi) : lat.volume * kk * kk / (2.0 * kPi * kPi);
            row_k.push_back(kk);
            row_w.push_back(density * kk * dl);
        }
    }

    // the last knot continues f smoothly: f_l = f, f_l' = f', f_l'' = f'' at r_c
    const int nk = 3 * R.n_knots, nfree = nk - 3;
    R.knots.assign(nk, 0.0);
    f.eval(rc, R.knots[nk - 3], R.knots[nk - 2], R.knots[nk - 1]);

    const size_t nrow = row_k.size();
    std::vector<double> design(nrow * nk), target(nrow);
    strided_threads(nrow, [&](size_t r) {
        double* d = &design[r * nk];
        knot_transforms(dim, R.n_knots, R.delta, row_k[r], d);
        // f_s's transform above k_cut is −(outside + Σ_free t_n d_n + Σ_fixed t_n d_n)
        double y = -f.outside(dim, rc, row_k[r]);
        for (int n = nfree; n < nk; ++n) y -= R.knots[n] * d[n];
        target[r] = y;
    });

    // weighted least squares by Givens rotations, one row at a time into the
    // triangular factor R and the rotated right-hand side z
    std::vector<double> tri(static_cast<size_t>(nfree) * nfree, 0.0), z(nfree, 0.0), a(nfree);
    for (size_t r = 0; r < nrow; ++r) {
        const double sw = std::sqrt(row_w[r]);
        for (int n = 0; n < nfree; ++n) a[n] = sw * design[r * nk + n];
        double rhs = sw * target[r];
        for (int j = 0; j < nfree; ++j) {
            if (a[j] == 0.0) continue;
            double* tj = &tri[static_cast<size_t>(j) * nfree];
            const double h = std::hypot(tj[j], a[j]);
            const double c = tj[j] / h, s = a[j] / h;
            tj[j] = h;
            a[j] = 0.0;
            for (int col = j + 1; col < nfree; ++col) {
                const double x = tj[col], y = a[col];
                tj[col] = c * x + s * y;
                a[col] = c * y - s * x;
            }
            const double x = z[j];
            z[j] = c * x + s * rhs;
            rhs = c * rhs - s * x;
        }
    }
    double dmax = 0.0, dmin = 0.0;
    for (int i = nfree - 1; i >= 0; --i) {
        const double rii = tri[static_cast<size_t>(i) * nfree + i];
        double s = z[i];
        for (int j = i + 1; j < nfree; ++j) s -= tri[static_cast<size_t>(i) * nfree + j] * R.knots[j];
        R.knots[i] = std::abs(rii) > 1e-300 ? s / rii : 0.0;
        if (std::abs(rii) > 1e-300) {
            dmax = std::max(dmax, std::abs(rii));
            dmin = dmin == 0.0 ? std::abs(rii) : std::min(dmin, std::abs(rii));
        }
    }
    R.condition = dmin > 0.0 ? dmax / dmin : 0.0;
    for (size_t r = 0; r < n_shell_rows; ++r) {
        double m = target[r];
        for (int n = 0; n < nfree; ++n) m -= R.knots[n] * design[r * nk + n];
        R.residual = std::max(R.residual, std::abs(m));
    }

    R.scaled.resize(nk);
    for (int n = 0; n < nk; ++n) R.scaled[n] = R.knots[n] * (n % 3 == 0 ? 1.0 : n % 3 == 1 ? R.delta : R.delta * R.delta);
    R.long_range_zero = R.knots[0];
    std::vector<double> d(nk);
    {
        knot_transforms(dim, R.n_knots, R.delta, 0.0, d.data());
        double s = f.inside(dim, rc, 0.0);
        for (int n = 0; n < nk; ++n) s -= R.knots[n] * d[n];
        R.short_range_k0 = s / lat.volume;
    }

    // retained vectors: one of each ±k pair (the first nonzero index
    // positive), |k| ≤ k_cut, in increasing index order; weight f̃_l(k)/V =
    // (outside + Σ t_n d_n) / V
    int nb[3];
    index_bounds(lat, R.k_cut, nb);
    int n[3];
    for (n[0] = 0; n[0] <= nb[0]; ++n[0])
        for (n[1] = -nb[1]; n[1] <= nb[1]; ++n[1])
            for (n[2] = -nb[2]; n[2] <= nb[2]; ++n[2]) {
                const bool upper = n[0] > 0 || (n[0] == 0 && (n[1] > 0 || (n[1] == 0 && n[2] > 0)));
                if (!upper) continue;
                double k[3];
                const double kk = kvector(lat, n, k);
                if (kk > R.k_cut || kk == 0.0) continue;
                knot_transforms(dim, R.n_knots, R.delta, kk, d.data());
                double w = f.outside(dim, rc, kk);
                for (int m = 0; m < nk; ++m) w += R.knots[m] * d[m];
                for (int i = 0; i < dim; ++i) {
                    R.n[i].push_back(n[i]);
                    R.kvec[i].push_back(k[i]);
                }
                R.weight.push_back(w / lat.volume);
            }
    return R;
}

}  // namespace alea_breakup
