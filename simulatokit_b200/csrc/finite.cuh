// finite.cuh -- shared declarations of the finite-projection builder (finite.cu) and its learned surrogate
// (surrogate.cu).
#pragma once

#include "context.cuh"

namespace simk {

constexpr int kGaussNodes = 48;     // Gauss-Legendre nodes on each side of u = 0
constexpr int kProfileRadii = 192;  // log-spaced radii of one (atom, slice) profile

// Scaled Lobato parameters of one element (LobatoParameterization.swift:38-44, exact pi).
struct ElementAB {
    double A[5], B[5];
};

// One atom's reach into one slice: the element (index into the potential's element list), the atom, the integration
// limits relative to the atom (zl < zu, both within +-R_c) and the atom's (x, y).
struct FinitePair {
    int elem, atom;
    double zl, zu, x, y;
};

struct FiniteSetup {
    std::vector<int> elements;        // distinct Z, ascending
    std::vector<ElementAB> ab;
    std::vector<double> rmin, rcut;   // per element
    std::vector<FinitePair> pairs;    // slice by slice
    std::vector<int> slice_first;     // pairs of slice j: [slice_first[j], slice_first[j + 1])
};

struct FiniteDevice {
    const FinitePair* pairs;
    const ElementAB* ab;
    const double* rmin;
    const double* rcut;
};

ElementAB element_ab(int z);
double finite_cutoff(int z);
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);
void ensure_gauss_nodes(Context& ctx);
FiniteSetup finite_setup(const GridGeom& g, const std::vector<double>& dz, int n_atoms, const int* Z, const double* xyz);
FiniteDevice upload_finite(Context& ctx, const FiniteSetup& s, DeviceBuffer& pairs, DeviceBuffer& ab,
                           DeviceBuffer& rmin, DeviceBuffer& rcut);
void finite_profiles_quadrature(Context& ctx, const FiniteDevice& d, long long npairs, int nr, double* table);
void finite_points(Context& ctx, const ElementAB* ab_dev, int n, const int* elem_dev, const double* rho_dev,
                   const double* zl_dev, const double* zu_dev, double* out_dev);
void finite_splat(Context& ctx, PotentialImpl& pot, const FiniteSetup& s, const FiniteDevice& d, int nr,
                  const double* table);
struct SurrogateImpl;
// V of every slice by finite projection: profiles by the surrogate where it was trained (judged by the quadrature on
// a sample; above `bound` the quadrature replaces it), by the float64 quadrature elsewhere; then the splat.
void build_potential_finite(Context& ctx, PotentialImpl& pot, int n_atoms, const int* Z, const double* xyz,
                            const SurrogateImpl* sg, double bound, int* used_surrogate, double* judged_max_rel);

}  // namespace simk
