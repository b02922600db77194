// Host-side compilation of the boundary configuration into the flat table the
// boundary kernel reads: FaceBC::FromConfig + PerFieldBC's constructor
// (src/face_bc.cpp:23-36, src/bcs/per_field_bc.cpp:188-243) plus the range
// resolution of FaceBC::Apply for a single rank that owns every face
// (src/face_bc.cpp:56-129).
#pragma once

#include <string>
#include <vector>

#include "../../include/mpd_b200.h"
#include "expr.hpp"
#include "lf_core.cuh"

namespace mpd {

struct CompiledBc {
    int nseg[4] = {0, 0, 0, 0};
    int first[4] = {0, 0, 0, 0};
    std::vector<SegDesc> seg;
    std::vector<int32_t> code;
    std::vector<double> consts;
};

// Boundary expression symbol names in BcSym order.
const std::vector<std::string> &BcSymbolNames();

// Returns an MPD_* status; on failure `err` holds a message in the
// reference's wording where the reference has one.
int CompileBc(const mpd_config &cfg, CompiledBc &out, std::string &err);

// ExpressionIC's eight programs (fields in IcSym order; NULL entries take
// the reference's defaults, src/ics/expression_ic.cpp:263-270) over the
// IcSym symbols, user constants folded in.  MPD_OK, MPD_ERR_INVALID (a user
// name shadows a built-in) or MPD_ERR_EXPR, with the reference's messages.
int CompileIc(const char *const exprs[8], int n_vars, const char *const *var_names,
              const double *var_values, ExprCode code[8], std::string &err);

// The first field (IcSym order, 0-7) whose expression reads a field of the
// same cell that is evaluated after it, or -1.  In the reference's one
// sequential sweep such a read sees the previous cell's value.
int IcForwardReference(const ExprCode code[8], int &read_field);

// Checks the grid sizes and pointers of a configuration (MPD_OK or MPD_ERR_INVALID).
int ValidateConfig(const mpd_config *cfg, const mpd_geometry *geom, std::string &err);

}  // namespace mpd
