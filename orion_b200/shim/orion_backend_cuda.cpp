// ORION's solver classes over the C ABI of the B200 path (see
// include/orion_backend_cuda.hpp for the contract).
//
// Built against the reference's own headers (-I <ORION>/src): every function
// below is a definition of a declaration the reference makes, with the
// reference's signature, so this file replaces src/solver/*.cpp and
// src/bc/PhysicalBC.cpp at link time.  It holds no numerics: each call binds
// the FlowFieldSet to a device case (orion_case_create), moves the host arrays
// the stage touches (coherent residency) and runs the stage's entry point.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "bc/PhysicalBC.hpp"
#include "solver/FluxComputer.hpp"
#include "solver/HaloExchanger.hpp"
#include "solver/InviscidFluxComputer.hpp"
#include "solver/ResidualMonitor.hpp"
#include "solver/StateUpdater.hpp"
#include "solver/TimeIntegrator.hpp"

#include "orion_backend_cuda.hpp"
#include "orion_gpu.h"

namespace orion::gpu {
namespace {

using preprocess::BlockField;
using preprocess::FlowFieldSet;

constexpr int kNg = 3;
enum : unsigned {
  kPrim = 1u << ORION_FIELD_PRIM,
  kQ = 1u << ORION_FIELD_Q,
  kDq = 1u << ORION_FIELD_DQ,
  kMetrics = 1u << ORION_FIELD_METRICS,
  kVol = 1u << ORION_FIELD_VOL,
  kDt = 1u << ORION_FIELD_DT,
  kC = 1u << ORION_FIELD_C,
  kMu = 1u << ORION_FIELD_MU,
  kAll = 0xffu,
};

struct Bound {
  orion_case_t h = nullptr;
  bool has_bc = false;
  bool has_params = false;
  orion_params_t params{};
  std::vector<int> nb;  // device block b <-> fs.blocks[nb[b]]
};

std::mutex g_mu;
std::unordered_map<const FlowFieldSet*, Bound> g_bound;
Residency g_mode = Residency::Coherent;
int g_precision = ORION_PREC_FP64;
bool g_device_ready = false;

[[noreturn]] void fail(const std::string& what) {
  throw std::runtime_error("orion_backend_cuda: " + what + ": " + orion_last_error());
}
void check(int rc, const char* what) {
  if (rc != ORION_OK) fail(what);
}

void ensure_device() {
  if (g_device_ready) return;
  const char* env = std::getenv("ORION_GPU_DEVICE");
  check(orion_gpu_init(env ? std::atoi(env) : 0), "orion_gpu_init");
  g_device_ready = true;
}

// core::Params -> the scalars the device path reads (Params.hpp:11-99; the
// derived freestream values are those init_inflow leaves, Inflow.cpp:300-459).
orion_params_t to_abi(const core::Params& p) {
  orion_params_t a{};
  a.gamma = p.inflow.gama;
  a.moo = p.inflow.moo;
  a.reynolds = p.inflow.reynolds;
  a.prl = p.inflow.prl;
  a.cfl = p.step.cfl;
  a.twall = p.inflow.twall;
  a.tref = p.inflow.tref;
  a.visc = p.inflow.visc;
  a.roo = p.inflow.roo;
  a.uoo = p.inflow.uoo;
  a.voo = p.inflow.voo;
  a.woo = p.inflow.woo;
  a.poo = p.inflow.poo;
  a.too = p.inflow.too;
  a.nvis = p.flowtype.nvis;
  a.method = p.control.method;
  a.ntmst = p.step.ntmst;
  a.csrv = p.technic.csrv;
  return a;
}

OrionArray<double>& field(BlockField& bf, int f) {
  switch (f) {
    case ORION_FIELD_PRIM: return bf.prim;
    case ORION_FIELD_Q: return bf.q;
    case ORION_FIELD_DQ: return bf.dq;
    case ORION_FIELD_METRICS: return bf.metrics;
    case ORION_FIELD_VOL: return bf.vol;
    case ORION_FIELD_DT: return bf.dt;
    case ORION_FIELD_C: return bf.c;
    default: return bf.mu;
  }
}

const int kNcomp[8] = {6, 5, 5, 9, 1, 1, 1, 1};

// Interior dims of a block from its padded vol array; checks every field's shape.
void block_dims(BlockField& bf, int nb, int dims[3]) {
  const auto& d = bf.vol.dims();
  if (d.size() != 3) throw std::runtime_error("orion_backend_cuda: block " + std::to_string(nb) + " not allocated");
  for (int a = 0; a < 3; ++a) dims[a] = (int)d[a] - 2 * kNg;
  const size_t npad = bf.vol.size();
  for (int f = 0; f < 8; ++f) {
    if (field(bf, f).size() != npad * kNcomp[f])
      throw std::runtime_error("orion_backend_cuda: block " + std::to_string(nb) + " field " + std::to_string(f) +
                               " does not have the padded shape (ng = 3)");
  }
}

void move(Bound& b, FlowFieldSet& fs, unsigned mask, bool up) {
  for (size_t i = 0; i < b.nb.size(); ++i) {
    BlockField& bf = fs.blocks[b.nb[i]];
    for (int f = 0; f < 8; ++f) {
      if (!(mask & (1u << f))) continue;
      double* p = field(bf, f).hostPtr();
      if (up) check(orion_case_upload(b.h, (int)i, f, p), "orion_case_upload");
      else check(orion_case_download(b.h, (int)i, f, p), "orion_case_download");
    }
  }
}

void set_params(Bound& b, const core::Params* p) {
  if (!p) return;
  const orion_params_t a = to_abi(*p);
  if (b.has_params && std::memcmp(&a, &b.params, sizeof(a)) == 0) return;
  check(orion_case_set_params(b.h, &a), "orion_case_set_params");
  b.params = a;
  b.has_params = true;
}

// The device case of fs, made (or remade with the BC regions, the first time
// a call brings them) from the host arrays.
Bound& bind(FlowFieldSet& fs, const bc::BCData* bc, const core::Params* p) {
  ensure_device();
  auto it = g_bound.find(&fs);
  if (it != g_bound.end() && bc && !it->second.has_bc) {
    // made by a call without BCData (regions unknown): remake with them
    if (g_mode == Residency::Resident) move(it->second, fs, kAll, false);
    check(orion_case_destroy(it->second.h), "orion_case_destroy");
    g_bound.erase(it);
    it = g_bound.end();
  }
  if (it == g_bound.end()) {
    if (fs.ng != kNg) throw std::runtime_error("orion_backend_cuda: ng must be 3");
    Bound b;
    b.nb = fs.local_block_ids;
    const int n = (int)b.nb.size();
    if (bc && bc->number_of_blocks != n)
      throw std::runtime_error("orion_backend_cuda: every block must be local to this process (one GPU, no sharding)");
    std::vector<std::vector<orion_region_t>> regs(n);
    std::vector<orion_block_desc_t> desc(n);
    for (int i = 0; i < n; ++i) {
      int dims[3];
      block_dims(fs.blocks[b.nb[i]], b.nb[i], dims);
      if (bc) {
        for (const auto& r : bc->block_bc[b.nb[i]].regions) {
          orion_region_t g{};
          for (int a = 0; a < 3; ++a) {
            g.s_st[a] = r.s_st[a];
            g.s_ed[a] = r.s_ed[a];
            g.t_st[a] = r.t_st[a];
            g.t_ed[a] = r.t_ed[a];
          }
          g.bctype = r.bctype;
          g.nbt = r.nbt;
          g.ibcwin = r.ibcwin;
          regs[i].push_back(g);
        }
      }
      desc[i].idim = dims[0];
      desc[i].jdim = dims[1];
      desc[i].kdim = dims[2];
      desc[i].nregions = (int)regs[i].size();
      desc[i].regions = regs[i].empty() ? nullptr : regs[i].data();
    }
    orion_params_t a{};
    if (p) a = to_abi(*p);
    check(orion_case_create(n, desc.data(), &a, g_precision, &b.h), "orion_case_create");
    b.has_bc = bc != nullptr;
    b.has_params = p != nullptr;
    b.params = a;
    try {
      move(b, fs, kAll, true);
    } catch (...) {
      orion_case_destroy(b.h);
      throw;
    }
    it = g_bound.emplace(&fs, std::move(b)).first;
  }
  set_params(it->second, p);
  return it->second;
}

// One stage: bind, move its inputs up, run it, move its outputs down.
template <class Launch>
Bound& stage(FlowFieldSet& fs, const bc::BCData* bc, const core::Params* p, unsigned in, unsigned out,
             const char* name, Launch&& launch) {
  Bound& b = bind(fs, bc, p);
  const bool coherent = g_mode == Residency::Coherent;
  if (coherent) move(b, fs, in & ~(kMetrics | kVol), true);
  check(launch(b.h), name);
  if (coherent) move(b, fs, out, false);
  return b;
}

}  // namespace

void set_residency(Residency mode) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_mode = mode;
}

void set_mixed_precision(bool mixed) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_precision = mixed ? ORION_PREC_MIXED : ORION_PREC_FP64;
}

void sync_to_host(preprocess::FlowFieldSet& fs) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_bound.find(&fs);
  if (it != g_bound.end()) move(it->second, fs, kAll, false);
}

void release(preprocess::FlowFieldSet& fs) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_bound.find(&fs);
  if (it == g_bound.end()) return;
  orion_case_destroy(it->second.h);
  g_bound.erase(it);
}

}  // namespace orion::gpu

void backend_cuda_init() {
  std::lock_guard<std::mutex> lk(orion::gpu::g_mu);
  orion::gpu::ensure_device();
  std::printf("[ORION] CUDA backend initialized (sm_100a)\n");
}

// ---------------------------------------------------------------------------
// The reference's declarations, defined on the device path.
// ---------------------------------------------------------------------------
namespace orion::solver {

using namespace orion::gpu;

void HaloExchanger::exchange_bc(bc::BCData& bc, preprocess::FlowFieldSet& fs) {
  std::lock_guard<std::mutex> lk(g_mu);
  stage(fs, &bc, nullptr, kPrim, kPrim, "exchange_bc", orion_exchange_bc);
}

void HaloExchanger::average_interface_residuals(bc::BCData& bc, preprocess::FlowFieldSet& fs) {
  std::lock_guard<std::mutex> lk(g_mu);
  stage(fs, &bc, nullptr, kDq, kDq, "average_interface_residuals", orion_average_interface_residuals);
}

void StateUpdater::update_flow_states(preprocess::FlowFieldSet& fs, const core::Params& params) {
  std::lock_guard<std::mutex> lk(g_mu);
  stage(fs, nullptr, &params, kPrim, kPrim | kC | kMu | kQ | kDq, "update_flow_states", orion_update_flow_states);
}

void StateUpdater::update_solution(preprocess::FlowFieldSet& fs, const bc::BCData& bc, const core::Params& params) {
  std::lock_guard<std::mutex> lk(g_mu);
  stage(fs, &bc, &params, kPrim | kMu | kDt | kDq, kPrim | kDq, "update_solution", orion_update_solution);
}

void TimeIntegrator::calculate_time_step(preprocess::FlowFieldSet& fs, core::Params& params) {
  std::lock_guard<std::mutex> lk(g_mu);
  Bound& b = stage(fs, nullptr, &params, kPrim | kC | kMu, kDt, "calculate_time_step", orion_calculate_time_step);
  check(orion_phydtime(b.h, &params.step.phydtime), "orion_phydtime");
}

void FluxComputer::compute_viscous_rhs(preprocess::FlowFieldSet& fs, const core::Params& params) {
  std::lock_guard<std::mutex> lk(g_mu);
  stage(fs, nullptr, &params, kPrim | kMu | kDq, kDq, "compute_viscous_rhs", orion_compute_viscous_rhs);
}

void InviscidFluxComputer::compute_inviscid_rhs(preprocess::FlowFieldSet& fs, const core::Params& params) {
  std::lock_guard<std::mutex> lk(g_mu);
  stage(fs, nullptr, &params, kPrim | kDq, kDq, "compute_inviscid_rhs", orion_compute_inviscid_rhs);
}

ResidualStats ResidualMonitor::compute(const preprocess::FlowFieldSet& fs, const core::Params& params) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto& mfs = const_cast<preprocess::FlowFieldSet&>(fs);  // read only: uploads copy from the host arrays
  orion_residual_t r{};
  Bound& b = stage(mfs, nullptr, &params, kDq | kDt, 0,
                   "ResidualMonitor::compute", [&](orion_case_t h) { return orion_residual_compute(h, &r); });
  ResidualStats s;
  s.rms_residual = r.rms;
  s.max_residual = r.max;
  s.max_loc[0] = b.nb[r.max_loc[0]];  // global block id, as ResidualMonitor.cpp:84
  for (int m = 1; m < 5; ++m) s.max_loc[m] = r.max_loc[m];
  return s;
}

}  // namespace orion::solver

namespace orion::bc {

void apply_physical_bc(const BCData& bc, preprocess::FlowFieldSet& fs, const core::Params& params) {
  std::lock_guard<std::mutex> lk(orion::gpu::g_mu);
  orion::gpu::stage(fs, &bc, &params, orion::gpu::kPrim, orion::gpu::kPrim, "apply_physical_bc",
                    orion_apply_physical_bc);
}

}  // namespace orion::bc
