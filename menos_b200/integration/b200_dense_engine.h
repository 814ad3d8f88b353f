// The reference-side binding's public surface (b200_dense_engine.cpp):
// what MENOS's registration (src/plan/execution_engines.cpp:24-31), its
// hardware profile (src/plan/hardware_profile.cpp) and a serving runtime call.
#pragma once

#include <cstdint>
#include <map>

#include "common/memory_ledger.h"
#include "mb2.h"
#include "menos/simulation_engine.h"
#include "plan/cuda_calibration.h"

namespace menos::engines::dense_b200 {

// The engine instance to register under (Engine::Dense, Backend::Cuda,
// Tier::InMemory), in place of the reference's CudaDenseEngine.
const SimulationEngine& b200_dense_engine();
// True when a device is usable (the registration's guard).
bool b200_device_available();
// The process's context on device 0 (opened on first use; NULL without a
// device), shared by every engine of this binding.
mb2_context* b200_context();
// The hardware profile's CUDA figures, measured on this engine (in place of
// plan::measure_cuda_calibration, src/plan/cuda_calibration.cpp:42-153).
plan::CudaCalibration measure_b200_calibration();

// The serving loop's admissions charged to a MemoryLedger
// (src/common/memory_ledger.h:37-117, Space::Device) for as long as each
// request holds its device memory, refused once the ledger's live device
// bytes would pass `device_limit` (0: no limit of its own -- the server's
// budget still applies).  A runtime keeps one per server:
//     ServerLedger hook(runtime_ledger, limit);
//     hook.attach(server);          // before the first mb2_server_submit
class ServerLedger {
public:
    ServerLedger(common::MemoryLedger& ledger, std::uint64_t device_limit) : ledger_(ledger), limit_(device_limit) {}
    ServerLedger(const ServerLedger&) = delete;
    ServerLedger& operator=(const ServerLedger&) = delete;
    int attach(mb2_server* server);

private:
    static int charge(void* user, std::uint64_t bytes);
    static void release(void* user, std::uint64_t bytes);
    common::MemoryLedger& ledger_;
    std::uint64_t limit_;
    std::multimap<std::uint64_t, common::MemoryLedger::Charge> live_;
};

}  // namespace menos::engines::dense_b200
