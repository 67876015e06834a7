// Optimized short-/long-range split of a periodic pair function.
//
// Natoli & Ceperley, J. Comput. Phys. 117, 171 (1995): a pair function f(r)
// summed over lattice images is written f = f_s + f_l, where f_l is a
// piecewise quintic Hermite function on [0, r_c] (value, slope and curvature
// at n_knots equally spaced knots; equal to f beyond r_c) chosen so that the
// Fourier transform of f_s = f − f_l is as small as possible above k_cut.
// The knot values minimise the χ² of that transform over the reciprocal
// lattice shells between k_cut and k_continuum, and over a continuum of k up
// to k_max weighted by the density of lattice vectors.  f_s then vanishes
// beyond r_c and is summed at the minimum image; f_l is summed over the
// retained vectors |k| ≤ k_cut.
//
// This module is the host side only: the device reads the knot table
// (`scaled`) and the retained vectors with their weights.
#pragma once

#include <memory>
#include <vector>

namespace alea_breakup {

// A lattice: rows a_i of the cell, reciprocal rows b_i (b_i · a_j = 2π δ_ij),
// cell volume (area in 2-D).  dim is 2 or 3.
struct Lattice {
    int dim = 2;
    double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double volume = 0.0;
};

// f(r) on (0, ∞): value and two r-derivatives, and the isotropic transforms
// of its pieces inside and outside r_c,
//   inside(k)  = ∫_{|r| < r_c} f e^{−ik·r} dᵈr,
//   outside(k) = ∫_{|r| > r_c} f e^{−ik·r} dᵈr.
class PairFunction {
public:
    virtual ~PairFunction() = default;
    virtual void eval(double r, double& f, double& df, double& d2f) const = 0;
    virtual double inside(int dim, double rc, double k) const;
    virtual double outside(int dim, double rc, double k) const = 0;
    double value(double r) const {
        double f, df, d2f;
        eval(r, f, df, d2f);
        return f;
    }

protected:
    // length scale below which f may vary (quadrature pieces are no wider)
    virtual double scale() const { return 0.0; }
};

// 1/r; its transforms are closed forms (2-D: 2π/k overall; 3-D: 4π/k²), and
// the 2-D outside transform is 2π/k minus the inside one.  `inner_floor` > 0
// leaves r < inner_floor · r_c out of the inside transform (and so puts it
// into the outside one).  The reference's geometric panels stop at
// r_c / 2⁴⁷, so its fit targets all carry −2π r_c 2⁻⁴⁷ (about −8e-12 at
// r_c = 172): a constant that the χ² fit turns into a 5e-6 relative shift of
// its tables at the largest k, where the targets themselves are ~1e-11.
// inner_floor = 2⁻⁴⁷ reproduces those tables to 1e-8; 0 gives the exact
// targets.
std::unique_ptr<PairFunction> coulomb(double inner_floor = 0.0);

// P(r)/Q(r) − lim_{r→∞} P/Q with P = Σ_{i≥1} num[i−1] rⁱ and
// Q = 1 + Σ_{i≥1} den[i−1] rⁱ (deg P ≤ deg Q, Q > 0 for r > 0; otherwise
// std::invalid_argument).  *limit receives lim P/Q.  The outside transform
// is integrated numerically between the zeros of the radial kernel and the
// alternating partial sums accelerated by Wynn's ε algorithm.
std::unique_ptr<PairFunction> rational(std::vector<double> num, std::vector<double> den, double* limit);

struct Options {
    int n_knots = 20;
    double k_cut = 0.0;        // 0: 8 |b|_min
    double k_continuum = 0.0;  // 0: 60 π / r_c
    double k_max = 0.0;        // 0: 6000 / r_c
    int n_continuum = 400;     // log-spaced midpoints on [k_continuum, k_max]
};

struct Result {
    int n_knots = 0;
    double rc = 0.0, delta = 0.0, k_cut = 0.0;
    std::vector<double> knots;    // [3·n_knots]: f_l, f_l', f_l'' at knot i
    std::vector<double> scaled;   // knots[3i + m] · delta^m (the device's table)
    // retained half-space vectors, |k| ≤ k_cut, and their weights f̃_l(k) / volume
    std::vector<int> n[3];
    std::vector<double> kvec[3], weight;
    double long_range_zero = 0.0;  // f_l(0)
    double short_range_k0 = 0.0;   // f̃_s(0) / volume
    double residual = 0.0;         // max over shell rows of the fit's misfit
    double condition = 0.0;        // max |R_jj| / min |R_jj| of the fit
};

Result optimize(const Lattice& lat, double rc, const PairFunction& f, const Options& opt);

}  // namespace alea_breakup
