// Host-side expression initial condition and one-shot expression evaluation
// (C ABI entry points mpd_expression_ic / mpd_eval_expression).
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/mpd_b200.h"
#include "bc_compile.hpp"
#include "expr.hpp"
#include "lf_core.cuh"

namespace mpd {
void SetLastError(const std::string &msg);
static const char *kIcNames[8] = {"rho", "v_z", "v_r", "v_phi", "H_z", "H_r", "H_phi", "e"};
}

using mpd::SetLastError;

namespace mpd {

int CompileIc(const char *const exprs[8], int n_vars, const char *const *var_names,
              const double *var_values, ExprCode code[8], std::string &err) {
    // ExpressionIC::Impl symbol table (src/ics/expression_ic.cpp:84-126)
    static const char *kReserved[] = {"gamma", "beta", "H_z0", "r_0", "z", "r", "r_z", "pi",
                                      "rho", "v_z", "v_r", "v_phi", "H_z", "H_r", "H_phi", "e"};
    const std::vector<std::string> syms = {"gamma", "beta", "H_z0", "r_0", "z", "r", "r_z",
                                           "rho", "v_z", "v_r", "v_phi", "H_z", "H_r", "H_phi", "e"};
    std::map<std::string, double> consts = {{"pi", M_PI}};
    for (int i = 0; i < n_vars; ++i) {
        const std::string name = var_names[i];
        for (const char *res : kReserved) {
            if (name == res) {
                err = "ExpressionIC: user variable '" + name + "' shadows the built-in symbol '" +
                      res + "'. Choose a different name.";
                return MPD_ERR_INVALID;
            }
        }
        if (consts.count(name)) {
            err = "ExpressionIC: failed to register user variable '" + name +
                  "' (name may already be taken by exprtk).";
            return MPD_ERR_INVALID;
        }
        consts[name] = var_values[i];
    }
    // defaults of src/ics/expression_ic.cpp:263-270, evaluation order
    static const char *kDefaults[8] = {"1.0", "0.0", "0.0", "0.0", "H_z0", "H_z * r_z",
                                       "(1 - 0.9 * z) * r_0 / r", "beta / (2 * (gamma - 1))"};
    for (int j = 0; j < 8; ++j) {
        const std::string src = (exprs && exprs[j]) ? exprs[j] : kDefaults[j];
        std::string perr;
        if (!CompileExpr(src, syms, consts, code[j], perr)) {
            err = std::string("ExpressionIC: failed to compile expression for '") + kIcNames[j] +
                  "':\n  expression : " + src + "\n  errors     :\n    [1] " + perr;
            return MPD_ERR_EXPR;
        }
    }
    return MPD_OK;
}

int IcForwardReference(const ExprCode code[8], int &read_field) {
    for (int j = 0; j < 8; ++j)
        for (int v : code[j].vars_used)
            if (v >= IC_F0 + j && v < IC_COUNT) {
                read_field = v - IC_F0;
                return j;
            }
    return -1;
}

}  // namespace mpd

extern "C" int mpd_expression_ic(const mpd_config *cfg, const mpd_geometry *geom,
                                 const char *const exprs[8], int n_vars,
                                 const char *const *var_names, const double *var_values,
                                 double *phys10_out) {
    std::string err;
    int rc = mpd::ValidateConfig(cfg, geom, err);
    if (rc == MPD_OK && (!geom || !phys10_out)) {
        err = "mpd_expression_ic: geometry and output are required";
        rc = MPD_ERR_INVALID;
    }
    if (rc != MPD_OK) {
        SetLastError(err);
        return rc;
    }
    mpd::ExprCode code[8];
    rc = mpd::CompileIc(exprs, n_vars, var_names, var_values, code, err);
    if (rc != MPD_OK) {
        SetLastError(err);
        return rc;
    }
    enum { S_GAMMA = mpd::IC_GAMMA, S_BETA = mpd::IC_BETA, S_HZ0 = mpd::IC_HZ0,
           S_R0 = mpd::IC_R0, S_Z = mpd::IC_Z, S_R = mpd::IC_R, S_RZ = mpd::IC_RZ,
           S_F0 = mpd::IC_F0 };
    const int L = cfg->L_max, M = cfg->M_max, rows = L + 2, cols = M + 3;
    const size_t n = static_cast<size_t>(rows) * cols;
    std::memset(phys10_out, 0, 10 * n * sizeof(double));
    double sym[S_F0 + 8] = {};
    sym[S_GAMMA] = cfg->gamma;
    sym[S_BETA] = cfg->beta;
    sym[S_HZ0] = cfg->H_z0;
    sym[S_R0] = cfg->r_0;
    const double gamma = cfg->gamma;
    // Output plane per evaluated field (Fields member order).
    const int plane_of[8] = {mpd::P_RHO, mpd::P_VZ, mpd::P_VR, mpd::P_VPHI,
                             mpd::P_HZ,  mpd::P_HR, mpd::P_HPHI, mpd::P_E};
    // ExpressionIC::Apply (src/ics/expression_ic.cpp:286-324): one sequential
    // sweep; field symbols keep their values between cells as in the reference.
    for (int l = 1; l < rows - 1; ++l) {
        const int l_global = l - 1;
        const double z = l_global * cfg->dz;
        const double rin = geom->r_inner[l], rout = geom->r_outer[l];
        const double drin = geom->dr_inner_dz[l], drout = geom->dr_outer_dz[l];
        for (int m = 1; m < cols - 1; ++m) {
            const int m_global = m - 1;
            const double frac = m_global * cfg->dy;
            sym[S_Z] = z;
            sym[S_R] = (1.0 - frac) * rin + frac * rout;
            sym[S_RZ] = (1.0 - frac) * drin + frac * drout;
            for (int j = 0; j < 8; ++j)
                sym[S_F0 + j] = mpd::eval_code(code[j].code.data(), code[j].consts.data(), sym);
            const size_t i = static_cast<size_t>(l) * cols + m;
            for (int j = 0; j < 8; ++j) phys10_out[plane_of[j] * n + i] = sym[S_F0 + j];
            const double rho = sym[S_F0 + 0], e = sym[S_F0 + 7];
            const double Hz = sym[S_F0 + 4], Hr = sym[S_F0 + 5], Hphi = sym[S_F0 + 6];
            const double p = (gamma - 1.0) * rho * e;
            phys10_out[mpd::P_PG * n + i] = p;
            phys10_out[mpd::P_PT * n + i] = p + 0.5 * (Hz * Hz + Hr * Hr + Hphi * Hphi);
        }
    }
    return MPD_OK;
}

extern "C" int mpd_eval_expression(const char *src, int n_syms, const char *const *names,
                                   const double *values, double *out) {
    if (!src || !out || n_syms < 0 || (n_syms > 0 && (!names || !values))) {
        SetLastError("mpd_eval_expression: bad arguments");
        return MPD_ERR_INVALID;
    }
    std::vector<std::string> syms;
    for (int i = 0; i < n_syms; ++i) syms.emplace_back(names[i]);
    mpd::ExprCode code;
    std::string perr;
    if (!mpd::CompileExpr(src, syms, {{"pi", M_PI}}, code, perr)) {
        SetLastError("expression '" + std::string(src) + "': " + perr);
        return MPD_ERR_EXPR;
    }
    *out = mpd::eval_code(code.code.data(), code.consts.data(), values);
    return MPD_OK;
}
