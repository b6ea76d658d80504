// surrogate.cuh -- the learned finite-projection profile (surrogate.cu).
#pragma once

#include "finite.cuh"

namespace simk {

constexpr int kEmbed = 16;
constexpr int kIn = kEmbed + 2;
constexpr int kHidden = 64;
constexpr int kSurrogateParams = 103 * kEmbed + kHidden * kIn + kHidden + 2 * (kHidden * kHidden + kHidden) + kHidden + 1;

struct SurrogateImpl {
    std::vector<int> elements;     // trained Z, ascending
    std::vector<double> rcut;      // per trained element
    double max_thickness = 4.0;    // the largest slab trained
    double rho_min = 0.01;         // the smallest radius trained
    double y_mean = 0.0, y_std = 1.0;  // the output is the fraction itself: kept at (0, 1)
    double train_loss = 0.0, val_max_rel = 0.0, val_rms_rel = 0.0;
    int steps = 0;
    long long samples = 0;
    DeviceBuffer params, grads, m, v;  // float32; inference stages f16 copies per block
    bool trained_on(int z) const {
        for (int e : elements)
            if (e == z) return true;
        return false;
    }
};

std::unique_ptr<SurrogateImpl> surrogate_train(Context& ctx, const std::vector<int>& elements, long long n_samples,
                                               int steps, int batch, double lr, unsigned long long seed,
                                               double max_thickness, double rho_min);
void surrogate_evaluate(Context& ctx, const SurrogateImpl& s, const std::vector<int>& z, const std::vector<double>& rho,
                        const std::vector<double>& zl, const std::vector<double>& zu, double* out_host);
void surrogate_quadrature_points(Context& ctx, const std::vector<int>& z, const std::vector<double>& rho,
                                 const std::vector<double>& zl, const std::vector<double>& zu, double* out_dev);
void surrogate_profiles(Context& ctx, const SurrogateImpl& s, const FiniteDevice& d, const int* pair_ids_dev,
                        int npairs, const int* elem_z_dev, const float2* rho_f0_dev, const double* pinf_dev, int nr,
                        double* table);
double surrogate_gradients(Context& ctx, SurrogateImpl& s, const std::vector<int>& z, const std::vector<double>& rho,
                           const std::vector<double>& zl, const std::vector<double>& zu,
                           const std::vector<double>& target, float* grads_host);
// The analytic infinite projection 2 sum_i [2 A_i/B_i K0(B_i rho) + A_i rho K1(B_i rho)] (host, float64).
double infinite_profile(int z, double rho);

}  // namespace simk
