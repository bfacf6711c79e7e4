// Versioned binary plan files (.cbplan): a built plan's host CB structures
// and device layouts, so a later process skips the CB build.  Host data only;
// a loaded plan is uploaded like a freshly built one.
#pragma once

#include <cstdint>
#include <string>

#include "cb_builder.hpp"
#include "cb_layout.hpp"

namespace cb {

// Everything a plan keeps on the host.  opts: the ten int fields of
// cbspmv_opts in declaration order.  flags & kPlanSpmvOnly: the file holds
// the host structures' scalars and the device layouts without their
// per-value arrays (enough to upload and multiply); counts: A's COO, CSR,
// DENSE and uniform blocks, segments and row patterns (what the plan's info
// reports), kept because such a file has no block arrays to count.
constexpr int32_t kPlanSpmvOnly = 1;
struct PlanImage {
    int32_t flags = 0;
    int32_t opts[10] = {};
    int32_t has_t = 0;
    int64_t counts[6] = {};
    HostCB *host = nullptr, *host_t = nullptr;
    DeviceLayout *A = nullptr, *AT = nullptr;
};

// Return "" or an error message.
std::string save_plan(const PlanImage &img, const std::string &path);
std::string load_plan(const std::string &path, PlanImage &img);

constexpr uint32_t kPlanFileVersion = 4;

}  // namespace cb
