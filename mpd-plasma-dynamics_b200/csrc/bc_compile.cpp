#include "bc_compile.hpp"

#include <cmath>
#include <map>

#include "expr.hpp"

namespace mpd {

const std::vector<std::string> &BcSymbolNames() {
    static const std::vector<std::string> names = {
        "gamma", "beta", "H_z0", "r_0", "dz", "dr", "r", "r_z", "z", "r_nb", "r_z_nb",
        "rho_nb", "v_z_nb", "v_r_nb", "v_phi_nb", "e_nb", "H_z_nb", "H_r_nb", "H_phi_nb",
        "rho", "v_z", "v_r", "v_phi", "H_z", "H_r", "H_phi", "e"};
    return names;
}

int ValidateConfig(const mpd_config *cfg, const mpd_geometry *geom, std::string &err) {
    if (!cfg) {
        err = "mpd_config is NULL";
        return MPD_ERR_INVALID;
    }
    if (cfg->L_max < 4 || cfg->M_max < 3) {
        err = "grid too small: need L_max >= 4 and M_max >= 3";
        return MPD_ERR_INVALID;
    }
    if (cfg->L_max > (1 << 20) || cfg->M_max > (1 << 20)) {
        err = "grid too large";
        return MPD_ERR_INVALID;
    }
    if (!(cfg->dz > 0.0) || !(cfg->dy > 0.0)) {
        err = "dz and dy must be positive";
        return MPD_ERR_INVALID;
    }
    if (cfg->precision != MPD_PRECISION_EXACT && cfg->precision != MPD_PRECISION_FAST) {
        err = "precision must be MPD_PRECISION_EXACT or MPD_PRECISION_FAST";
        return MPD_ERR_INVALID;
    }
    if (geom && (!geom->r_inner || !geom->r_outer || !geom->dr_inner_dz || !geom->dr_outer_dz)) {
        err = "mpd_geometry has a NULL profile";
        return MPD_ERR_INVALID;
    }
    for (int f = 0; f < 4; ++f) {
        if (cfg->n_segments[f] < 0 || (cfg->n_segments[f] > 0 && !cfg->segments[f])) {
            err = "bad segment list";
            return MPD_ERR_INVALID;
        }
    }
    return MPD_OK;
}

namespace {

const char *kEvalNames[8] = {"rho", "v_z", "v_r", "v_phi", "H_z", "H_r", "H_phi", "e"};

// Conditions of a segment in evaluation order.
void EvalOrder(const mpd_bc_segment &s, const mpd_field_cond *out[8]) {
    out[Q_RHO] = &s.rho;
    out[Q_VZ] = &s.v_z;
    out[Q_VR] = &s.v_r;
    out[Q_VPHI] = &s.v_phi;
    out[Q_HZ] = &s.H_z;
    out[Q_HR] = &s.H_r;
    out[Q_HPHI] = &s.H_phi;
    out[Q_E] = &s.e;
}

// Symbols that are the same in every cell: their values are known here.
bool CellIndependent(int sym) {
    return sym == BS_GAMMA || sym == BS_BETA || sym == BS_HZ0 || sym == BS_R0 || sym == BS_DZ;
}

double CellIndependentValue(const mpd_config &cfg, int sym) {
    switch (sym) {
        case BS_GAMMA: return cfg.gamma;
        case BS_BETA: return cfg.beta;
        case BS_HZ0: return cfg.H_z0;
        case BS_R0: return cfg.r_0;
        default: return cfg.dz;
    }
}

// Closed form of a compiled expression (SegDesc::form and operands of field
// j).  Folding evaluates the same IEEE operations in the same order as the
// interpreter would, so every form gives the interpreter's bits.
void ClosedForm(const mpd_config &cfg, const ExprCode &ec, int j, SegDesc &d) {
    d.form[j] = EF_GENERAL;
    d.fa[j] = d.fb[j] = -1;
    d.ca[j] = d.cb[j] = 0.0;
    d.fop[j] = OP_MUL;
    bool foldable = true;
    for (int32_t ins : ec.code) {
        const int op = ins & 0xff;
        const int arg = ins >> 8;
        const bool arith = op == OP_END || op == OP_CONST || op == OP_NEG || op == OP_ADD ||
                           op == OP_SUB || op == OP_MUL || op == OP_DIV;
        if (!(arith || (op == OP_VAR && CellIndependent(arg)))) foldable = false;
    }
    if (foldable) {
        double sym[BS_COUNT];
        for (int t = 0; t < BS_COUNT; ++t) sym[t] = CellIndependent(t) ? CellIndependentValue(cfg, t) : NAN;
        d.form[j] = EF_CONST;
        d.ca[j] = eval_code(ec.code.data(), ec.consts.data(), sym);
        return;
    }
    // operand: a symbol (cell-independent ones become constants) or a constant
    auto operand = [&](int32_t ins, int &sym, double &c) {
        const int op = ins & 0xff;
        const int arg = ins >> 8;
        if (op == OP_CONST) {
            sym = -1;
            c = ec.consts[arg];
            return true;
        }
        if (op != OP_VAR) return false;
        if (CellIndependent(arg)) {
            sym = -1;
            c = CellIndependentValue(cfg, arg);
        } else {
            sym = arg;
        }
        return true;
    };
    const std::vector<int32_t> &c = ec.code;
    if (c.size() == 2 && (c[1] & 0xff) == OP_END && operand(c[0], d.fa[j], d.ca[j])) {
        // x * 1.0 is x exactly
        d.form[j] = EF_BIN;
        d.fop[j] = OP_MUL;
        d.fb[j] = -1;
        d.cb[j] = 1.0;
        return;
    }
    if (c.size() == 4 && (c[3] & 0xff) == OP_END) {
        const int op = c[2] & 0xff;
        if ((op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_DIV) &&
            operand(c[0], d.fa[j], d.ca[j]) && operand(c[1], d.fb[j], d.cb[j])) {
            d.form[j] = EF_BIN;
            d.fop[j] = op;
            return;
        }
    }
    d.fa[j] = d.fb[j] = -1;
}

}  // namespace

int CompileBc(const mpd_config &cfg, CompiledBc &out, std::string &err) {
    out = CompiledBc();
    const int L = cfg.L_max, M = cfg.M_max;
    const std::map<std::string, double> consts = {{"pi", M_PI}};
    int total = 0;
    for (int f = 0; f < 4; ++f) total += cfg.n_segments[f];
    if (total > kMaxSegments) {
        err = "too many boundary segments (max " + std::to_string(kMaxSegments) + ")";
        return MPD_ERR_UNSUPPORTED_BC;
    }
    for (int f = 0; f < 4; ++f) {
        out.first[f] = static_cast<int>(out.seg.size());
        out.nseg[f] = cfg.n_segments[f];
        const bool l_face = f == FACE_L_LO || f == FACE_L_HI;
        const int face_hi = l_face ? M : L - 1;  // FaceGlobalRange
        for (int k = 0; k < cfg.n_segments[f]; ++k) {
            const mpd_bc_segment &sc = cfg.segments[f][k];
            const mpd_field_cond *c[8];
            EvalOrder(sc, c);
            SegDesc d{};
            bool has_axis = false;
            for (int j = 0; j < 8; ++j) {
                if (c[j]->type < MPD_NEUMANN || c[j]->type > MPD_AXIS_LF) {
                    err = "unknown field condition type";
                    return MPD_ERR_INVALID;
                }
                if (c[j]->type == MPD_AXIS_LF) has_axis = true;
            }
            // PerFieldBC constructor validation (src/bcs/per_field_bc.cpp:211-233)
            if (has_axis && f != FACE_M_LO) {
                err = "PerFieldBC: AxisLF condition is only valid on the M_LO face "
                      "(inner boundary / axis of symmetry)";
                return MPD_ERR_INVALID;
            }
            const int no_axis[4] = {Q_VR, Q_VPHI, Q_HR, Q_HPHI};
            for (int j : no_axis) {
                if (c[j]->type == MPD_AXIS_LF) {
                    err = std::string("PerFieldBC: AxisLF is only valid for rho, v_z, e, and H_z "
                                      "(fields with a defined half-stencil LF update).  '") +
                          kEvalNames[j] +
                          "' has no AxisLF formula.  Use { dirichlet: 0.0 } for symmetry "
                          "components that must be zero.";
                    return MPD_ERR_INVALID;
                }
            }
            d.has_axis = has_axis ? 1 : 0;
            for (int j = 0; j < 8; ++j) {
                d.type[j] = c[j]->type;
                d.value[j] = c[j]->value;
                d.code[j] = -1;
                if (c[j]->type != MPD_EXPRESSION) continue;
                const std::string src = c[j]->expr ? c[j]->expr : "";
                ExprCode ec;
                std::string perr;
                if (!CompileExpr(src, BcSymbolNames(), consts, ec, perr)) {
                    err = std::string("PerFieldBC: failed to compile BC expression for field '") +
                          kEvalNames[j] + "':\n  expression : " + src +
                          "\n  error(s)   :\n    [1] " + perr;
                    return MPD_ERR_EXPR;
                }
                // A field may read the boundary values of fields evaluated
                // before it in the same cell.  Reading itself or a later
                // field sees the previous cell's leftover in the reference
                // (src/bcs/per_field_bc.cpp:29-32): order-dependent, so the
                // parallel device path refuses it.
                for (int v : ec.vars_used) {
                    if (v >= BS_CUR0 && v - BS_CUR0 >= j) {
                        err = std::string("expression for '") + kEvalNames[j] + "' reads '" +
                              kEvalNames[v - BS_CUR0] +
                              "', which is evaluated at or after it (forward reference; the "
                              "reference leaves its value from the previous cell): not supported";
                        return MPD_ERR_UNSUPPORTED_BC;
                    }
                }
                ClosedForm(cfg, ec, j, d);
                // relocate constants into the shared pool
                const int cbase = static_cast<int>(out.consts.size());
                out.consts.insert(out.consts.end(), ec.consts.begin(), ec.consts.end());
                d.code[j] = static_cast<int>(out.code.size());
                for (int32_t ins : ec.code) {
                    const int op = ins & 0xff;
                    if (op == OP_CONST) ins = ((((ins >> 8) + cbase)) << 8) | OP_CONST;
                    out.code.push_back(ins);
                }
            }
            // FaceBC::Apply range resolution, ClipToLocal (owned range is the
            // whole face) and the M_LO corner policy (src/face_bc.cpp:110-124)
            const int g_lo = sc.global_lo < 0 ? 0 : sc.global_lo;
            const int g_hi = sc.global_hi < 0 ? face_hi : sc.global_hi;
            const int clo = g_lo > 0 ? g_lo : 0;
            const int chi = g_hi < face_hi ? g_hi : face_hi;
            int lo = clo + 1, hi = chi + 1;
            if (clo > chi) {
                lo = 1;
                hi = 0;
            } else if (f == FACE_M_LO) {
                if (lo < 2) lo = 2;
                if (hi > L - 1) hi = L - 1;
            }
            d.lo = lo;
            d.hi = hi;
            out.seg.push_back(d);
        }
    }
    if (out.code.empty()) out.code.push_back(OP_END);
    if (out.consts.empty()) out.consts.push_back(0.0);
    return MPD_OK;
}

}  // namespace mpd
