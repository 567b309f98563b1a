// Launch wrappers around the reference's own hot-path kernels.
//
// TEST INFRASTRUCTURE ONLY: the golden-fixture driver (oracle/_ref/pkref_driver)
// that runs PhysIKA's kernels on a GPU to pin the CPU restatement. Nothing in
// the product links it.
//
// Each wrapper lives in the translation unit that includes the reference
// source file defining its kernels (refk_<part>.cu), and launches them with
// the arguments, launch shape (BLOCK_SIZE = 64 threads, cudaGridSize blocks)
// and order of the reference host method it names. The kernels are the
// reference's; the launch code is ours.
#pragma once
#include "prelude.h"
#include "Core/Array/Array.h"
#include "Core/DataTypes.h"
#include "Framework/Topology/NeighborList.h"
#include "Dynamics/ParticleSystem/NeighborData.h"
#include <vector>

namespace PhysIKA {
template <typename TDataType> class GridHash;
}

namespace refk {
typedef PhysIKA::DataType3f DT;
typedef float Real;
typedef PhysIKA::Vector3f Coord;
typedef PhysIKA::Matrix3f Matrix;
typedef PhysIKA::TPair<DT> NPair;
template <typename T> using DArr = PhysIKA::DeviceArray<T>;
template <typename T> using NList = PhysIKA::NeighborList<T>;

// GridHash::construct (Framework/Topology/GridHash.cu:297-323) with checks: the
// reduced particle count and the scanned cell offsets are compared with a host
// computation before the kernel that writes at those offsets runs.
void grid_construct(PhysIKA::GridHash<DT>& hash, DArr<Coord>& pos);
void checked_count_and_scan(int* d_counts, int num, int reduced, const char* what);
void checked_offsets(int* d_offsets, const std::vector<int>& counts, const char* what);
std::vector<int> download_ints(int* d, int num);

// NeighborQuery (Framework/Topology/NeighborQuery.cu): the grid hash is set up
// as NeighborQuery::initializeImpl does (GridHash::setSpace(h, lo, hi), :107-149),
// then built and queried as compute() does (:152-199): queryNeighborFixed
// (:584-605) when cap > 0, else queryNeighborDynamic (:450-478). The list is
// resized as the reference's NeighborField would size it. Returns the number of
// elements. n must be a multiple of 64: the three query kernels guard with
// `pId > size` (:253,345,524), so a grid with threads past n would let thread n
// read and write one entry past the arrays; a grid of exactly n threads has no
// such thread.
int neighbor_query(DArr<Coord>& pos, Real h, Coord lo, Coord hi, int cap, NList<int>& nbr);

// SummationDensity::compute(rho, pos, nbr, h, mass) (SummationDensity.cu:96-110):
// K_ComputeDensity with mass = m_factor * m_particle_mass.
void summation_density(DArr<Real>& rho, DArr<Coord>& pos, NList<int>& nbr, Real h, Real mass);
// calculateScalingFactor (SummationDensity.cu:112-138) evaluated with the
// reference's SpikyKernel<float>::Weight; returns m_factor, sets *mass.
Real density_factor(Real sampling, Real h, Real rho0, Real* mass);

// DensityPBD::takeOneIteration (DensityPBD.cu:305-365), the variant without
// per-particle inverse mass: reset dpos, density, K_ComputeLambdas,
// K_ComputeDisplacement, K_UpdatePosition.
void pbd_iteration(DArr<Coord>& pos, DArr<Coord>& vel, NList<int>& nbr, DArr<Real>& rho,
                   DArr<Real>& lambda, DArr<Coord>& dpos, Real h, Real dt, Real mass);
// DensityPBD::updateVelocity (DensityPBD.cu:380-392): DP_UpdateVelocity.
void pbd_update_velocity(DArr<Coord>& vel, DArr<Coord>& pos_old, DArr<Coord>& pos, Real dt);

// ParticleIntegrator::begin's force reset and integrate() (ParticleIntegrator.cu:
// 19-34, 84-138): K_UpdateVelocity(vel, force, gravity, dt), K_UpdatePosition.
void integrate(DArr<Coord>& pos, DArr<Coord>& vel, DArr<Coord>& force, Coord g, Real dt);

// ElasticityModule (Dynamics/ParticleSystem/ElasticityModule.cu):
// resetRestShape (:496-517, K_UpdateRestShape), computeInverseK (:390-401,
// EM_PrecomputeShape), one enforceElasticity (:342-369: reset, EM_EnforceElasticity,
// K_UpdatePosition) and updateVelocity (:423-437, K_UpdateVelocity).
void pd_rest_shape(NList<NPair>& shape, NList<int>& nbr, DArr<Coord>& pos);
void pd_inverse_k(DArr<Matrix>& invK, NList<NPair>& shape, Real horizon);
void pd_enforce(DArr<Coord>& pos, DArr<Coord>& pos_old, DArr<Coord>& disp, DArr<Real>& weights,
                DArr<Real>& bulk, DArr<Matrix>& invK, NList<NPair>& shape, Real horizon, Real mu,
                Real lambda);
void pd_update_velocity(DArr<Coord>& vel, DArr<Coord>& pos_old, DArr<Coord>& pos, Real dt);
}  // namespace refk
