// Internal to the library: the error slot behind `qm_last_error` and the line-level table, for
// the translation units whose C entry points run on the host only.
#pragma once

#include <string>
#include <vector>

#include "../../include/qm_batch.h"

namespace qm {

// Sets the calling thread's last error and returns `status`.
qm_status set_error(qm_status status, const std::string &message);
// The calling thread's last error.
const std::string &last_error();
// The line-level quantile table (41 x 100 floats), built by its seeded simulation on first use.
const std::vector<float> &line_level_table_shared();

}  // namespace qm
