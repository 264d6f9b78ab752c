// Oracle driver for the UNMODIFIED ORION reference solver.  TEST INFRASTRUCTURE ONLY.
//
// Reads a case directory written by orion_b200.cases (param.dat, grid.x in
// Plot3D Fortran-sequential form, bc.inp in ORION's BC format), runs the
// reference's own set-up functions in the order of OrionSolver::preprocess
// (src/core/OrionSolver.cpp:32-100, minus the MPI distributors, which are
// no-ops on one rank), applies the seeded initial noise, then replays the
// per-step stage sequence of OrionSolver::solve (src/core/OrionSolver.cpp:139-209)
// WITHOUT the debug block at :156-201 (it calls MPI_Abort after the first
// viscous RHS, so the reference driver itself can never take a second step).
//
// Usage:
//   orion_ref_harness <case_dir> <nsteps> <out_dir> [--snap-step S] [--time-only]
//                     [--warmup W]
// Writes <out_dir>/init.bin, final.bin (field states), hist.bin (residual
// history) and, with --snap-step S, snap_S_<stage>.bin after every stage of
// step S.  With --time-only it prints the step-loop wall time and writes
// nothing but hist.bin.  --warmup W runs W untimed steps before the timed ones.
#include <mpi.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "bc/BCPreprocess.hpp"
#include "bc/BCReader.hpp"
#include "bc/PhysicalBC.hpp"
#include "core/Params.hpp"
#include "core/Runtime.hpp"
#include "mesh/MetricComputer.hpp"
#include "mesh/Plot3DReader.hpp"
#include "preprocess/FlowField.hpp"
#include "preprocess/Inflow.hpp"
#include "preprocess/InitialCondition.hpp"
#include "postprocess/PostProcess.hpp"
#include "solver/FluxComputer.hpp"
#include "solver/HaloExchanger.hpp"
#include "solver/InviscidFluxComputer.hpp"
#include "solver/ResidualMonitor.hpp"
#include "solver/StateUpdater.hpp"
#include "solver/TimeIntegrator.hpp"
#ifdef ORION_SHIM
#include "orion_backend_cuda.hpp"
#endif

using namespace orion;

namespace {

// splitmix64: the seeded noise generator shared by every path that builds an
// initial state (orion_b200.cases implements the same sequence).
struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

void write_arr(std::ofstream& f, const OrionArray<double>& a) {
  f.write(reinterpret_cast<const char*>(a.hostPtr()), (std::streamsize)(a.size() * sizeof(double)));
}

// Field-state file: header, then per block prim(6) q(5) dq(5) metrics(9) vol dt c mu
// spec(3) specv(3), each an i-fastest padded array exactly as OrionArray stores it.
void dump_state(const std::string& path, const preprocess::FlowFieldSet& fs, double phydtime) {
  std::ofstream f(path, std::ios::binary);
  const char magic[8] = {'O', 'R', 'S', 'T', 'A', 'T', 'E', '1'};
  f.write(magic, 8);
  int32_t hdr[3] = {(int32_t)fs.local_block_ids.size(), fs.ng, 0};
  f.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
  f.write(reinterpret_cast<const char*>(&phydtime), sizeof(double));
  for (int nb : fs.local_block_ids) {
    const auto& bf = fs.blocks[nb];
    int32_t d[3] = {(int32_t)bf.prim.dims()[0], (int32_t)bf.prim.dims()[1], (int32_t)bf.prim.dims()[2]};
    f.write(reinterpret_cast<const char*>(d), sizeof(d));
  }
  for (int nb : fs.local_block_ids) {
    const auto& bf = fs.blocks[nb];
    write_arr(f, bf.prim);
    write_arr(f, bf.q);
    write_arr(f, bf.dq);
    write_arr(f, bf.metrics);
    write_arr(f, bf.vol);
    write_arr(f, bf.dt);
    write_arr(f, bf.c);
    write_arr(f, bf.mu);
    write_arr(f, bf.spec_radius);
    write_arr(f, bf.spec_radius_visc);
  }
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <case_dir> <nsteps> <out_dir> [--snap-step S] [--time-only] [--warmup W] [--vts FLOWNAME]\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const int nsteps = std::atoi(argv[2]);
  const std::string out = argv[3];
  int snap_step = -1;
  bool time_only = false;
  int warmup = 0;
  std::string vts;  // --vts FLOWNAME: the reference's own solution output after the run
  for (int a = 4; a < argc; ++a) {
    std::string s = argv[a];
    if (s == "--snap-step" && a + 1 < argc) snap_step = std::atoi(argv[++a]);
    else if (s == "--time-only") time_only = true;
    else if (s == "--warmup" && a + 1 < argc) warmup = std::atoi(argv[++a]);
    else if (s == "--vts" && a + 1 < argc) vts = argv[++a];
#ifdef ORION_SHIM
    else if (s == "--resident") orion::gpu::set_residency(orion::gpu::Residency::Resident);
    else if (s == "--mixed") orion::gpu::set_mixed_precision(true);
#endif
  }
#ifdef ORION_SHIM
  // The same driver over the B200 path: the solver classes resolve to
  // orion_b200/shim/orion_backend_cuda.cpp instead of the reference's TUs.
  backend_cuda_init();
#endif

  core::Runtime::init(argc, argv);

  core::Params params;
  params.load_namelist_file(dir + "/param.dat");

  // Noise spec: seed and amplitude, written beside the case by the case builder.
  uint64_t seed = 0;
  double amp = 0.0;
  {
    std::ifstream nf(dir + "/noise.txt");
    if (nf) nf >> seed >> amp;
  }

  // --- OrionSolver::preprocess (src/core/OrionSolver.cpp:32-100), one rank ---
  mesh::MultiBlockGrid grid = mesh::Plot3DReader::read(dir + "/grid.x", params.inflow.ndim);
  bc::BCData bcd = bc::BCReader::read_parallel_bc_root_only(dir + "/bc.inp", grid, 1, {.mbsmarker = 1976, .verbose = false});
  bc::set_bc_index(bcd);
  bc::prepare_bc_topology(bcd);
  preprocess::FlowFieldSet fs = preprocess::allocate_other_variable(grid, bcd, params, 5, 6);
  preprocess::fill_bc_flag(grid, bcd, fs);
  mesh::compute_grid_metrics(grid, fs, params);
  mesh::check_grid_metrics(grid, fs, bcd);
  preprocess::init_inflow(params, fs);
  preprocess::initialize_flow(params, fs);

  // Seeded noise on rho and u over every padded point, blocks in order, k,j,i order.
  if (amp != 0.0) {
    SplitMix64 rng{seed};
    for (int nb : fs.local_block_ids) {
      auto& bf = fs.blocks[nb];
      const int nx = (int)bf.prim.dims()[0], ny = (int)bf.prim.dims()[1], nz = (int)bf.prim.dims()[2];
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            double r1 = rng.uniform();
            double r2 = rng.uniform();
            bf.prim(i, j, k, 0) = bf.prim(i, j, k, 0) * (1.0 + amp * (2.0 * r1 - 1.0));
            bf.prim(i, j, k, 1) = bf.prim(i, j, k, 1) * (1.0 + amp * (2.0 * r2 - 1.0));
          }
    }
  }
  preprocess::update_temperature(params, fs);

  if (!time_only) dump_state(out + "/init.bin", fs, params.step.phydtime);

  solver::HaloExchanger halo;
  std::vector<double> hist;  // per step: rms, max, loc[5], phydtime
  hist.reserve((size_t)nsteps * 8);

  auto snap = [&](int step, const char* name) {
#ifdef ORION_SHIM
    if (step == snap_step) orion::gpu::sync_to_host(fs);
#endif
    if (step == snap_step) dump_state(out + "/snap_" + std::to_string(step) + "_" + name + ".bin", fs, params.step.phydtime);
  };

  auto t0 = std::chrono::steady_clock::now();
  for (int step = -warmup; step < nsteps; ++step) {
    if (step == 0) t0 = std::chrono::steady_clock::now();
    snap(step, "pre");
    halo.exchange_bc(bcd, fs);
    snap(step, "exchange");
    bc::apply_physical_bc(bcd, fs, params);
    snap(step, "bc");
    solver::StateUpdater::update_flow_states(fs, params);
    snap(step, "state");
    solver::TimeIntegrator::calculate_time_step(fs, params);
    snap(step, "dt");
    if (params.flowtype.nvis == 1) {
      solver::FluxComputer::compute_viscous_rhs(fs, params);
      snap(step, "visc");
      halo.average_interface_residuals(bcd, fs);
      snap(step, "avg1");
    }
    solver::InviscidFluxComputer::compute_inviscid_rhs(fs, params);
    snap(step, "inv");
    halo.average_interface_residuals(bcd, fs);
    snap(step, "avg2");
    solver::StateUpdater::update_solution(fs, bcd, params);
    snap(step, "update");
    auto rs = solver::ResidualMonitor::compute(fs, params);
    if (step < 0) continue;
    hist.push_back(rs.rms_residual);
    hist.push_back(rs.max_residual);
    for (int m = 0; m < 5; ++m) hist.push_back((double)rs.max_loc[m]);
    hist.push_back(params.step.phydtime);
  }
  auto t1 = std::chrono::steady_clock::now();
  double secs = std::chrono::duration<double>(t1 - t0).count();

  {
    std::ofstream f(out + "/hist.bin", std::ios::binary);
    int32_t n = nsteps;
    f.write(reinterpret_cast<const char*>(&n), sizeof(n));
    f.write(reinterpret_cast<const char*>(hist.data()), (std::streamsize)(hist.size() * sizeof(double)));
  }
#ifdef ORION_SHIM
  orion::gpu::sync_to_host(fs);
#endif
  if (!time_only) dump_state(out + "/final.bin", fs, params.step.phydtime);
  if (!vts.empty()) {
    params.filename.flowname = vts;
    postprocess::PostProcess::write_solution(fs, grid, params, nsteps);
  }

  long long pts = 0;
  for (int nb : fs.local_block_ids) pts += (long long)grid.blocks[nb].npoints();
  std::printf("{\"steps\": %d, \"seconds\": %.6f, \"points\": %lld, \"pt_steps_per_s\": %.6e}\n",
              nsteps, secs, pts, nsteps > 0 ? (double)pts * nsteps / secs : 0.0);
  return 0;
}
