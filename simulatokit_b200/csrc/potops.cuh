// potops.cuh -- operations on a built potential: tiling (ProjectedPotential.tiled) and projection
// (ProjectedPotential.project), on the device.
#pragma once

#include "context.cuh"

namespace simk {

// ProjectedPotential.tiled(repetitionsX:repetitionsY:repetitionsZ:) (ProjectedPotential.swift:76-105): `out` gets
// every slice of `src` tiled rx x ry times in the plane (extent multiplied, sampling kept) and the whole stack repeated
// rz times. Refuses, before allocating, counts below 1, a tiled slice of more than 2^28 values, more than 1,000,000
// slices and more than 2^31 values in all.
void tile_potential(Context& ctx, const PotentialImpl& src, long long rx, long long ry, long long rz,
                    PotentialImpl& out);

// ProjectedPotential.project() (ProjectedPotential.swift:64-73): out_dev[i] = sum over slices in order of V[s][i].
void project_potential(Context& ctx, const PotentialImpl& p, double* out_dev);

}  // namespace simk
