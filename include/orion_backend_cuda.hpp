/* C++ drop-in layer: ORION's solver classes on the B200 path.
 *
 * orion_b200/shim/orion_backend_cuda.cpp defines, over the C ABI of
 * orion_gpu.h, the reference's own declarations of
 *   orion::solver::InviscidFluxComputer::compute_inviscid_rhs  (InviscidFluxComputer.hpp:17-18)
 *   orion::solver::FluxComputer::compute_viscous_rhs           (FluxComputer.hpp:15-16)
 *   orion::solver::TimeIntegrator::calculate_time_step         (TimeIntegrator.hpp:10-11)
 *   orion::solver::StateUpdater::update_flow_states            (StateUpdater.hpp:14-15)
 *   orion::solver::StateUpdater::update_solution               (StateUpdater.hpp:21-23)
 *   orion::solver::HaloExchanger::exchange_bc                  (HaloExchanger.hpp:20-21)
 *   orion::solver::HaloExchanger::average_interface_residuals  (HaloExchanger.hpp:25)
 *   orion::solver::ResidualMonitor::compute                    (ResidualMonitor.hpp:20-21)
 *   orion::bc::apply_physical_bc                               (PhysicalBC.hpp:17-19)
 * so a driver written against src/solver links against this layer instead of
 * those seven translation units, unchanged.  The declarations below are the
 * additions of this layer; they need none of the reference's headers.
 *
 * Residency.  Each FlowFieldSet gets one device case, made at its first call.
 *  - Coherent (default): every call uploads the host arrays the stage reads and
 *    downloads those it writes, so host and device agree after every call and a
 *    driver may read or modify the host arrays between calls.
 *  - Resident: the host arrays are uploaded once, at the first call; later calls
 *    work on the device copy only.  sync_to_host() brings every field back.
 * In both modes metrics and vol are uploaded at the first call only (they are
 * set-up data); call release() after changing them.  spec_radius and
 * spec_radius_visc are not written: the time step is fused with its spectra.
 *
 * Errors: a failing call throws std::runtime_error carrying orion_last_error(),
 * the reference's own error convention (OrionArray.hpp:25-27).
 */
#pragma once

namespace orion {
namespace preprocess {
struct FlowFieldSet;
}
namespace gpu {

enum class Residency { Coherent, Resident };

/* Applies to FlowFieldSets bound after the call. */
void set_residency(Residency mode);
/* Precision of the device cases made after the call: false = plain FP64 (the
 * default, bit-identical to the reference), true = the mixed FP32/FP64 path. */
void set_mixed_precision(bool mixed);
/* Downloads every field of fs's device case into fs's host arrays (waits). */
void sync_to_host(preprocess::FlowFieldSet& fs);
/* Frees fs's device case; the next call makes a new one from the host arrays. */
void release(preprocess::FlowFieldSet& fs);

}  // namespace gpu
}  // namespace orion

/* The backend hook: selects the CUDA device (ORION_GPU_DEVICE, default 0). The
 * reference's CPU hook is backend_cpu_init() (src/backend/cpu/BackendCPU.cpp:3). */
void backend_cuda_init();
