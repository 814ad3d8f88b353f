// The reference-side binding of the noisy engines (b200_noisy_engines.cpp):
// the density-matrix and trajectory engines of MENOS
// (src/engines/density_matrix, src/engines/trajectory) on the device, as
// menos::SimulationEngine instances a registration adds beside the
// reference's CPU ones.
#pragma once

#include "menos/simulation_engine.h"

namespace menos::engines::dense_b200 {

// (Engine::DensityMatrix, Backend::Cuda, Tier::InMemory): rho on the device,
// bitwise the reference DensityMatrixEngine's; identical counts (readout
// errors included) and Factorized draws; traces within 1e-12.
const SimulationEngine& b200_density_matrix_engine();
// (Engine::Trajectory, Backend::Cuda, Tier::InMemory): each trajectory's
// state the reference TrajectoryEngine's; identical counts, term means within
// 1e-12.
const SimulationEngine& b200_trajectory_engine();

}  // namespace menos::engines::dense_b200
