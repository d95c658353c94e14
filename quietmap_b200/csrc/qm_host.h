// Internal to the library: the error slot behind `qm_last_error`, for the translation units whose
// C entry points run on the host only (qm_formats.cpp).
#pragma once

#include <string>

#include "../../include/qm_batch.h"

namespace qm {

// Sets the calling thread's last error and returns `status`.
qm_status set_error(qm_status status, const std::string &message);
// The calling thread's last error.
const std::string &last_error();

}  // namespace qm
