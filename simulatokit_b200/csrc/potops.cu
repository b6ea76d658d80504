// potops.cu -- tiling and projection of a built potential on the device (ProjectedPotential.swift:64-105).
//
// Tiling a unit cell's potential replaces building a large periodic crystal atom by atom: the crystal's slices are
// the cell's, repeated in the plane and along the beam, so one cell is built and the copies are a memory-bound
// gather. Both kernels copy or add float64 values in the reference's order, so their results are the reference's bits.
#include <algorithm>

#include "potops.cuh"

namespace simk {

namespace {

inline int blocks_for(long long n, int threads = 256) {
    return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 16));
}

// One output row (slice s', x index X) a block at a time: out[(s' MX + X) MY + Y] = V[((s' mod S) nx + X mod nx) ny +
// Y mod ny]. Rows are read once from L2 (the source is small) and written once, coalesced.
__global__ void k_tile_slices(const double* __restrict__ V, int S, int nx, int ny, int MX, int MY, long long rows,
                              double* __restrict__ out) {
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const long long sp = row / MX;
        const int X = (int)(row - sp * MX);
        const double* src = V + ((sp % S) * nx + X % nx) * (long long)ny;
        double* dst = out + row * MY;
        int y = threadIdx.x % ny;
        const int step = blockDim.x % ny;
        for (int Y = threadIdx.x; Y < MY; Y += blockDim.x) {
            dst[Y] = __ldg(src + y);
            y += step;
            if (y >= ny) y -= ny;
        }
    }
}

// out[i] = ((0 + V[0][i]) + V[1][i]) + ..., slices in order.
__global__ void k_project(const double* __restrict__ V, int S, long long N, double* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int s = 0; s < S; ++s) acc = __dadd_rn(acc, V[s * N + i]);
        out[i] = acc;
    }
}

}  // namespace

void tile_potential(Context& ctx, const PotentialImpl& src, long long rx, long long ry, long long rz,
                    PotentialImpl& out) {
    const std::string refusal = "repetitions must be at least 1 along every axis and give at most 2^28 values a "
                                "slice, 1,000,000 slices and 2^31 values in all, got (" + std::to_string(rx) + ", " +
                                std::to_string(ry) + ", " + std::to_string(rz) + ")";
    SIMK_REQUIRE(rx >= 1 && ry >= 1 && rz >= 1, refusal);
    const long long S = src.n_slices();
    // every product checked against its bound before the next can overflow
    SIMK_REQUIRE(rz <= 1000000 && S * rz <= 1000000, refusal);
    SIMK_REQUIRE(rx <= (1LL << 28) && ry <= (1LL << 28), refusal);
    const long long mx = (long long)src.g.nx * rx, my = (long long)src.g.ny * ry;
    SIMK_REQUIRE(mx <= (1LL << 28) && my <= (1LL << 28) && mx * my <= (1LL << 28), refusal);
    const long long per_slice = mx * my, slices = S * rz;
    SIMK_REQUIRE(per_slice * slices <= (1LL << 31), refusal);
    out.ctx = &ctx;
    out.g.nx = (int)mx;
    out.g.ny = (int)my;
    out.g.ex = src.g.ex * (double)rx;
    out.g.ey = src.g.ey * (double)ry;
    out.dz.clear();
    for (long long r = 0; r < rz; ++r) out.dz.insert(out.dz.end(), src.dz.begin(), src.dz.end());
    out.V.alloc((size_t)(per_slice * slices) * sizeof(double));
    out.t_energy = -1.0;
    const long long rows = slices * mx;
    {
        KernelTimer t(ctx, "tile", 8.0 * (double)(per_slice * slices) + 8.0 * (double)(S * src.g.count()));
        k_tile_slices<<<(int)std::min<long long>(rows, (long long)ctx.sm_count * 16), 256, 0, ctx.stream>>>(
            src.V.as<double>(), (int)S, src.g.nx, src.g.ny, (int)mx, (int)my, rows, out.V.as<double>());
    }
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
}

void project_potential(Context& ctx, const PotentialImpl& p, double* out_dev) {
    const long long N = p.g.count();
    k_project<<<blocks_for(N), 256, 0, ctx.stream>>>(p.V.as<double>(), p.n_slices(), N, out_dev);
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
}

}  // namespace simk
