// Solver_Config JSON reader (the reference schema of json_Files/Solver_Config.json, read by the
// reference with jsoncpp at src/Configuration_Read.cpp:23-87).  A small recursive-descent parser
// that accepts // and /* */ comments as jsoncpp does by default.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cfd_b200.h"

namespace cfdb {

struct JVal {
  enum Kind { NUL, BOOL, NUM, STR, OBJ, ARR } kind = NUL;
  double num = 0.0;
  bool b = false;
  std::string str;
  std::map<std::string, std::shared_ptr<JVal>> obj;
  std::vector<std::shared_ptr<JVal>> arr;
  const JVal *get(const std::string &k) const {
    auto it = obj.find(k);
    return it == obj.end() ? nullptr : it->second.get();
  }
};

namespace {
struct Parser {
  const std::string &s;
  size_t i = 0;
  std::string err;
  explicit Parser(const std::string &src) : s(src) {}
  void ws() {
    for (;;) {
      while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) i++;
      if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '/') {
        while (i < s.size() && s[i] != '\n') i++;
      } else if (i + 1 < s.size() && s[i] == '/' && s[i + 1] == '*') {
        size_t e = s.find("*/", i + 2);
        i = (e == std::string::npos) ? s.size() : e + 2;
      } else {
        return;
      }
    }
  }
  bool fail(const std::string &m) {
    if (err.empty()) err = m + " at offset " + std::to_string(i);
    return false;
  }
  bool str(std::string &out) {
    if (i >= s.size() || s[i] != '"') return fail("expected string");
    i++;
    out.clear();
    while (i < s.size() && s[i] != '"') {
      if (s[i] == '\\' && i + 1 < s.size()) {
        i++;
        char c = s[i];
        out.push_back(c == 'n' ? '\n' : c == 't' ? '\t' : c);
      } else {
        out.push_back(s[i]);
      }
      i++;
    }
    if (i >= s.size()) return fail("unterminated string");
    i++;
    return true;
  }
  bool value(JVal &v) {
    ws();
    if (i >= s.size()) return fail("unexpected end");
    char c = s[i];
    if (c == '{') {
      v.kind = JVal::OBJ;
      i++;
      ws();
      if (i < s.size() && s[i] == '}') {
        i++;
        return true;
      }
      for (;;) {
        ws();
        std::string k;
        if (!str(k)) return false;
        ws();
        if (i >= s.size() || s[i] != ':') return fail("expected ':'");
        i++;
        auto child = std::make_shared<JVal>();
        if (!value(*child)) return false;
        v.obj[k] = child;
        ws();
        if (i < s.size() && s[i] == ',') {
          i++;
          ws();
          if (i < s.size() && s[i] == '}') {  // trailing comma
            i++;
            return true;
          }
          continue;
        }
        if (i < s.size() && s[i] == '}') {
          i++;
          return true;
        }
        return fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.kind = JVal::ARR;
      i++;
      ws();
      if (i < s.size() && s[i] == ']') {
        i++;
        return true;
      }
      for (;;) {
        auto child = std::make_shared<JVal>();
        if (!value(*child)) return false;
        v.arr.push_back(child);
        ws();
        if (i < s.size() && s[i] == ',') {
          i++;
          continue;
        }
        if (i < s.size() && s[i] == ']') {
          i++;
          return true;
        }
        return fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.kind = JVal::STR;
      return str(v.str);
    }
    if (s.compare(i, 4, "true") == 0) {
      v.kind = JVal::BOOL;
      v.b = true;
      i += 4;
      return true;
    }
    if (s.compare(i, 5, "false") == 0) {
      v.kind = JVal::BOOL;
      v.b = false;
      i += 5;
      return true;
    }
    if (s.compare(i, 4, "null") == 0) {
      v.kind = JVal::NUL;
      i += 4;
      return true;
    }
    const char *start = s.c_str() + i;
    char *end = nullptr;
    double d = std::strtod(start, &end);
    if (end == start) return fail("bad value");
    v.kind = JVal::NUM;
    v.num = d;
    i += static_cast<size_t>(end - start);
    return true;
  }
};

bool as_double(const JVal *v, double &out) {
  if (!v) return false;
  if (v->kind == JVal::NUM) out = v->num;
  else if (v->kind == JVal::BOOL) out = v->b ? 1.0 : 0.0;
  else return false;
  return true;
}
bool as_int(const JVal *v, int &out) {
  double d;
  if (!as_double(v, d)) return false;
  out = static_cast<int>(d);
  return true;
}
bool as_bool(const JVal *v, int &out) {
  double d;
  if (!as_double(v, d)) return false;
  out = d != 0.0 ? 1 : 0;
  return true;
}
int enum_from(const JVal *v, const std::vector<std::string> &names, int dflt) {
  if (!v) return dflt;
  if (v->kind == JVal::NUM) return static_cast<int>(v->num);
  if (v->kind == JVal::STR) {
    std::string u;
    for (char ch : v->str) u.push_back(static_cast<char>(std::tolower(static_cast<unsigned char>(ch))));
    for (size_t k = 0; k < names.size(); k++)
      if (u == names[k]) return static_cast<int>(k);
  }
  return dflt;
}
}  // namespace

bool parse_json(const std::string &text, JVal &root, std::string &err) {
  Parser p(text);
  if (!p.value(root)) {
    err = p.err;
    return false;
  }
  return true;
}

std::string config_from_json(const std::string &text, cfd_config *cfg) {
  JVal root;
  std::string err;
  if (!parse_json(text, root, err)) return err;
  if (root.kind != JVal::OBJ) return "top level is not an object";
  const JVal *sim = root.get("Simulation");
  const JVal *sol = root.get("Solver");
  const JVal *lim = root.get("LimiterCoefficients");
  const JVal *bc = root.get("BoundaryConditions");
  if (sim) as_double(sim->get("CFL"), cfg->cfl);
  if (sol) {
    as_int(sol->get("Dissipation_Type"), cfg->dissipation_type);
    as_bool(sol->get("Is_Second_Order"), cfg->is_second_order);
    as_bool(sol->get("Time_Accurate"), cfg->time_accurate);
    as_bool(sol->get("Local_Time_Stepping"), cfg->local_time_stepping);
    as_bool(sol->get("Is_WENO"), cfg->weno);
    as_bool(sol->get("Is_Char"), cfg->weno_characteristic);
    as_bool(sol->get("Is_MOVERS_1"), cfg->movers_single_alpha);
    as_bool(sol->get("Enable_Entropy_Fix"), cfg->movers_entropy_fix);
    const JVal *fs = sol->get("Flux_Scheme");
    if (fs && fs->kind == JVal::STR) {
      int k = enum_from(fs, {"llf", "roe", "ausm", "hllc", "ausm_gpu", "movers", "ricca", "movers_nwsc"}, -1);
      const int map[8] = {CFD_DISS_LLF,      CFD_DISS_ROE,    CFD_DISS_AUSM,  CFD_DISS_HLLC,
                          CFD_DISS_AUSM_GPU, CFD_DISS_MOVERS, CFD_DISS_RICCA, CFD_DISS_MOVERS_NWSC};
      if (k >= 0) cfg->dissipation_type = map[k];
    }
    cfg->limiter = enum_from(sol->get("Limiter_Type"), {"minmod_reference", "minmod", "vanleer", "superbee", "vanalbada"},
                             cfg->limiter);
    cfg->integrator = enum_from(sol->get("Integrator"), {"reference", "rk4", "ssprk3", "rk3_gpu_ref", "rk4_gpu_ref"},
                                cfg->integrator);
    cfg->precision = enum_from(sol->get("Precision"), {"fp64", "fp32_flux"}, cfg->precision);
    cfg->reconstruct_primitive = enum_from(sol->get("Reconstruction"), {"conserved", "primitive"}, cfg->reconstruct_primitive);
    as_int(sol->get("Reorder"), cfg->reorder);
    cfg->muscl = enum_from(sol->get("MUSCL"), {"reference", "gradient"}, cfg->muscl);
    as_double(sol->get("Entropy_Fix_Linear"), cfg->entropy_fix_linear);
    as_double(sol->get("Shock_Fix"), cfg->shock_fix);
  }
  if (lim) {
    as_double(lim->get("Limiter_Zeta"), cfg->limiter_zeta);
    as_double(lim->get("Limiter_Zeta1"), cfg->limiter_zeta1);
  }
  if (bc) {
    cfg->inlet_bc = enum_from(bc->get("Inlet_BC"), {"supersonic", "subsonic_reference", "total_pt", "fixed", "farfield"},
                             cfg->inlet_bc);
    cfg->exit_bc = enum_from(bc->get("Exit_BC"), {"supersonic", "subsonic_reference", "static_p"}, cfg->exit_bc);
    int sub = 0;
    if (as_bool(bc->get("Is_Inlet_SubSonic"), sub)) cfg->inlet_bc = sub ? CFD_INLET_SUBSONIC_REF : CFD_INLET_SUPERSONIC;
    if (as_bool(bc->get("Is_Exit_SubSonic"), sub)) cfg->exit_bc = sub ? CFD_EXIT_SUBSONIC_REF : CFD_EXIT_SUPERSONIC;
    as_double(bc->get("Inlet_Rho"), cfg->inlet_rho);
    as_double(bc->get("Inlet_P"), cfg->inlet_p);
    as_double(bc->get("Inlet_u"), cfg->inlet_u);
    as_double(bc->get("Inlet_v"), cfg->inlet_v);
    as_double(bc->get("Inlet_P0"), cfg->inlet_p0);
    as_double(bc->get("Inlet_T0"), cfg->inlet_t0);
    as_double(bc->get("Exit_P"), cfg->exit_p);
    as_double(bc->get("R_Gas"), cfg->r_gas);
  }
  return "";
}

}  // namespace cfdb
