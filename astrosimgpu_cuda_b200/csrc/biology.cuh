// biology.cuh -- named access to the model's biology parameters and the JSON
// override loader (a flat object of parameter names to values).
#pragma once

#include <string>

#include "common.cuh"
#include "model.cuh"

namespace astrosim {

// Applies a JSON object such as {"exc_poiss_rate": 3000, "stp_enabled": false}
// to `bio`.  Names are the fields of Biology (the reference's constants,
// src/astrosim_fused.cu:742-781); numbers for the real and integer fields,
// true / false (or 0 / 1) for the flags.  NULL or an empty / blank string changes
// nothing.  Unknown names, repeated names, malformed text and values that the
// model cannot run with are errors that name the problem.
Status apply_biology_json(const char* json, Biology& bio);

// Comma-separated list of every parameter name.
std::string biology_names();

// Value of one parameter of `bio` as a double (flags as 0 / 1).
Status biology_get(const Biology& bio, const char* name, double* value);

}  // namespace astrosim
