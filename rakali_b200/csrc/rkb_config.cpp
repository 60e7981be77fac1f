// Namelist parsing and validation (see rkb_config.hpp).
#include "rkb_config.hpp"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <functional>
#include <map>
#include <set>
#include <vector>

namespace rkb {
namespace {

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// One value token of a namelist record.
struct Tok {
  enum Kind { kName, kEq, kComma, kValue, kLParen, kRParen } kind;
  std::string text;
  bool quoted = false;
};

// Tokenise a group body.  Strings keep their content; '!' starts a comment
// outside strings.
bool tokenize(const std::string& body, std::vector<Tok>& out, std::string& err) {
  size_t i = 0, n = body.size();
  while (i < n) {
    char c = body[i];
    if (std::isspace((unsigned char)c)) { ++i; continue; }
    if (c == '!') {
      while (i < n && body[i] != '\n') ++i;
      continue;
    }
    if (c == '=') { out.push_back({Tok::kEq, "="}); ++i; continue; }
    if (c == ',') { out.push_back({Tok::kComma, ","}); ++i; continue; }
    if (c == '(') { out.push_back({Tok::kLParen, "("}); ++i; continue; }
    if (c == ')') { out.push_back({Tok::kRParen, ")"}); ++i; continue; }
    if (c == '\'' || c == '"') {
      char q = c;
      std::string s;
      ++i;
      bool closed = false;
      while (i < n) {
        if (body[i] == q) {
          if (i + 1 < n && body[i + 1] == q) { s += q; i += 2; continue; }
          closed = true;
          ++i;
          break;
        }
        s += body[i++];
      }
      if (!closed) { err = "unterminated string"; return false; }
      Tok t{Tok::kValue, s};
      t.quoted = true;
      out.push_back(t);
      continue;
    }
    size_t j = i;
    while (j < n && !std::isspace((unsigned char)body[j]) && body[j] != '=' && body[j] != ',' &&
           body[j] != '!' && body[j] != '(' && body[j] != ')')
      ++j;
    std::string word = body.substr(i, j - i);
    // A bare word followed (after spaces) by '=' or '(' is a key name.
    size_t k = j;
    while (k < n && (body[k] == ' ' || body[k] == '\t')) ++k;
    bool is_name = (std::isalpha((unsigned char)word[0]) || word[0] == '_') &&
                   k < n && (body[k] == '=' || body[k] == '(') && word[0] != '.';
    out.push_back({is_name ? Tok::kName : Tok::kValue, word});
    i = j;
  }
  return true;
}

bool parse_real(const std::string& raw, double& v) {
  std::string s = lower(raw);
  for (auto& c : s)
    if (c == 'd' || c == 'q') c = 'e';
  // Fortran kind suffix such as 1.0_wp or 1.0_8
  auto us = s.find('_');
  if (us != std::string::npos) s = s.substr(0, us);
  if (s.empty()) return false;
  char* end = nullptr;
  v = std::strtod(s.c_str(), &end);
  return end && *end == '\0' && std::isfinite(v);
}

bool parse_int(const std::string& raw, int& v) {
  std::string s = raw;
  auto us = s.find('_');
  if (us != std::string::npos) s = s.substr(0, us);
  if (s.empty()) return false;
  char* end = nullptr;
  long x = std::strtol(s.c_str(), &end, 10);
  if (!end || *end != '\0') return false;
  v = (int)x;
  return true;
}

bool parse_bool(const std::string& raw, bool& v) {
  std::string s = lower(trim(raw));
  if (!s.empty() && s[0] == '.') s = s.substr(1);
  if (s.empty()) return false;
  if (s[0] == 't') { v = true; return true; }
  if (s[0] == 'f') { v = false; return true; }
  return false;
}

enum class Kind { Int, Real, Bool, Str, RealArr, Any };

struct Key {
  Kind kind;
  std::function<void(Config&, const std::vector<std::string>&, int index)> set;  // may be empty
};

using Schema = std::map<std::string, std::map<std::string, Key>>;

// Every group/key of build_rakali_schema (rki_config.F90:1234-1800).  Keys the
// 2D step uses get setters; the rest are accepted and ignored (Kind::Any).
const Schema& schema() {
  static Schema S = [] {
    Schema s;
    auto any = [&](const char* g, std::initializer_list<const char*> keys) {
      for (auto k : keys) s[g][k] = Key{Kind::Any, {}};
    };
#define RK_INT(g, k, field) \
  s[g][#k] = Key{Kind::Int, [](Config& c, const std::vector<std::string>& v, int) { parse_int(v[0], c.field); }}
#define RK_REAL(g, k, field) \
  s[g][#k] = Key{Kind::Real, [](Config& c, const std::vector<std::string>& v, int) { parse_real(v[0], c.field); }}
#define RK_BOOL(g, k, field) \
  s[g][#k] = Key{Kind::Bool, [](Config& c, const std::vector<std::string>& v, int) { parse_bool(v[0], c.field); }}
#define RK_STR(g, k, field) \
  s[g][#k] = Key{Kind::Str, [](Config& c, const std::vector<std::string>& v, int) { c.field = v[0]; }}
    RK_STR("sim", sim_type, sim_type);
    RK_STR("grid", grid_type, grid_type);
    RK_INT("grid", nx, nx);
    RK_INT("grid", ny, ny);
    RK_REAL("grid", dx, dx);
    RK_REAL("grid", dy, dy);
    RK_INT("grid", nghost, nghost);
    RK_REAL("time", t_end, t_end);
    RK_REAL("time", cfl, cfl);
    RK_REAL("time", dt_max, dt_max);
    RK_REAL("time", dt_fixed, dt_fixed);
    RK_INT("time", cfl_interval, cfl_interval);
    RK_STR("time", time_scheme, time_scheme);
    RK_STR("time", time_unit, time_unit);
    any("si", {"precond", "rtol", "wetdry", "wetdry_nsub", "wetdry_bsub_fill", "newton_max",
               "newton_tol"});
    any("metadata", {"reference_time", "institution"});
    RK_STR("logging", log_level, log_level);
    any("logging", {"status_interval"});
    any("vcoord", {"vcoord_type", "remap_method", "vcoord_depth_transition",
                   "vcoord_blend_width", "zstar_h_surf_target", "zstar_stretching",
                   "zstar_h_min", "zstar_n_surf", "rho_ref_pressure", "rho_target_light",
                   "rho_target_dense"});
    RK_REAL("physics", manning_n, manning_n);
    RK_REAL("physics", dry_threshold, dry_threshold);
    RK_REAL("physics", wind_stress_x, wind_stress_x);
    RK_REAL("physics", wind_stress_y, wind_stress_y);
    RK_REAL("physics", coriolis_f, coriolis_f);
    RK_BOOL("physics", use_hllc, use_hllc);
    RK_BOOL("physics", use_linear_bottom_drag, use_linear_bottom_drag);
    RK_REAL("physics", bottom_drag_r, bottom_drag_r);
    RK_BOOL("physics", wind_surface_layer, wind_surface_layer);
    any("output", {"output_to_file", "output_dir", "output_interval", "output_format",
                   "restart_interval", "async_output", "async_buffer_slots", "compress_output",
                   "compress_level", "restart_file", "forcing_file", "forcing_x_origin",
                   "forcing_y_origin", "gauge_file", "gauge_output_interval", "out_h_layer",
                   "out_velocity", "out_salinity", "out_temperature", "out_density", "out_w"});
    RK_STR("output", bathymetry_file, bathymetry_file);
    RK_STR("boundary", bc_west, bc_west);
    RK_STR("boundary", bc_east, bc_east);
    RK_STR("boundary", bc_south, bc_south);
    RK_STR("boundary", bc_north, bc_north);
    RK_REAL("boundary", tidal_amplitude, tidal_amplitude);
    RK_REAL("boundary", tidal_period, tidal_period);
    RK_INT("boundary", n_tidal_constituents, n_tidal_constituents);
    s["boundary"]["tidal_amp"] = Key{Kind::RealArr, [](Config& c, const std::vector<std::string>& v, int idx) {
      for (size_t k = 0; k < v.size() && idx + (int)k < kMaxTidalCfg; ++k) parse_real(v[k], c.tidal_amp[idx + k]);
    }};
    s["boundary"]["tidal_phase"] = Key{Kind::RealArr, [](Config& c, const std::vector<std::string>& v, int idx) {
      for (size_t k = 0; k < v.size() && idx + (int)k < kMaxTidalCfg; ++k) parse_real(v[k], c.tidal_phase[idx + k]);
    }};
    s["boundary"]["tidal_omega"] = Key{Kind::RealArr, [](Config& c, const std::vector<std::string>& v, int idx) {
      for (size_t k = 0; k < v.size() && idx + (int)k < kMaxTidalCfg; ++k) parse_real(v[k], c.tidal_omega[idx + k]);
    }};
    RK_REAL("boundary", inflow_velocity, inflow_velocity);
    RK_REAL("boundary", inflow_salinity, inflow_salinity);
    RK_REAL("boundary", inflow_temperature, inflow_temperature);
    RK_REAL("boundary", discharge_flux, discharge_flux);
    RK_REAL("boundary", clamped_elevation, clamped_elevation);
    RK_INT("boundary", sponge_width, sponge_width);
    RK_REAL("boundary", sponge_strength, sponge_strength);
    RK_REAL("boundary", sponge_h_ref, sponge_h_ref);
    RK_STR("boundary", nesting_file, nesting_file);
    any("boundary", {"nesting_x_origin", "nesting_y_origin"});
    any("tracer", {"initial_salinity", "s_ref", "beta_s", "s_min", "s_max", "kappa_s_bg",
                   "s_init_surface", "s_init_bottom", "initial_temperature", "t_ref", "alpha_t",
                   "t_min", "t_max", "kappa_t_bg", "eos_form", "t_init_surface",
                   "t_init_bottom", "tracer_recon", "use_sediment", "sediment_w_s",
                   "sediment_initial_conc", "sediment_bed_init", "sediment_tau_crit_erosion",
                   "sediment_erosion_rate", "sediment_porosity"});
    RK_BOOL("tracer", use_ppm_tracer, use_ppm_tracer);
    RK_STR("initial_condition", init_condition, init_condition);
    RK_REAL("initial_condition", eta_initial, eta_initial);
    RK_REAL("initial_condition", h0, h0);
    RK_REAL("initial_condition", hump_amplitude, hump_amplitude);
    RK_REAL("initial_condition", hump_sigma, hump_sigma);
    RK_REAL("initial_condition", hump_x_offset, hump_x_offset);
    RK_REAL("initial_condition", hump_y_offset, hump_y_offset);
    RK_REAL("initial_condition", init_u_shear, init_u_shear);
    RK_BOOL("nonhydrostatic", use_nonhydrostatic, use_nonhydrostatic);
    RK_INT("nonhydrostatic", nz_layers, nz_layers);
    RK_BOOL("nonhydrostatic", use_multilayer, use_multilayer);
    any("nonhydrostatic", {"nh_tolerance", "nh_max_iterations", "nh_preconditioner",
                           "nh_solve_interval", "split_ratio", "split_averaging", "rho_0",
                           "vmix_nu_max", "vmix_nu_bg", "vmix_ri_alpha", "vmix_use_kpp",
                           "vmix_use_keps", "keps_si_picard", "kpp_ri_crit",
                           "kpp_cs_nonlocal", "kpp_c_vt2", "hdiff_kappa", "smagorinsky_cs",
                           "biharmonic_nu4", "evap_mass_sink", "evap_latent_cooling",
                           "ml_min_depth", "bpg_method", "keps_stability"});
#undef RK_INT
#undef RK_REAL
#undef RK_BOOL
#undef RK_STR
    return s;
  }();
  return S;
}

bool check_value(Kind k, const std::vector<std::string>& vals, const std::vector<bool>& quoted) {
  if (vals.empty()) return false;
  switch (k) {
    case Kind::Int: { int x; return vals.size() == 1 && !quoted[0] && parse_int(vals[0], x); }
    case Kind::Real: { double x; return vals.size() == 1 && !quoted[0] && parse_real(vals[0], x); }
    case Kind::Bool: { bool x; return vals.size() == 1 && !quoted[0] && parse_bool(vals[0], x); }
    case Kind::Str: return vals.size() == 1;
    case Kind::RealArr:
      for (size_t i = 0; i < vals.size(); ++i) {
        double x;
        if (quoted[i] || !parse_real(vals[i], x)) return false;
      }
      return true;
    default: return true;
  }
}

// Expand Fortran repeat counts ("3*1.0").
void expand_repeat(std::vector<std::string>& vals, std::vector<bool>& quoted) {
  std::vector<std::string> v2;
  std::vector<bool> q2;
  for (size_t i = 0; i < vals.size(); ++i) {
    const std::string& s = vals[i];
    auto star = s.find('*');
    int n = 0;
    if (!quoted[i] && star != std::string::npos && parse_int(s.substr(0, star), n) && n > 0) {
      for (int k = 0; k < n; ++k) {
        v2.push_back(s.substr(star + 1));
        q2.push_back(false);
      }
    } else {
      v2.push_back(s);
      q2.push_back(quoted[i]);
    }
  }
  vals.swap(v2);
  quoted.swap(q2);
}

}  // namespace

bool parse_namelist(const std::string& text, Config& cfg, std::string& err) {
  const Schema& S = schema();
  size_t pos = 0, n = text.size();
  while (pos < n) {
    // find the next '&' outside comments
    size_t amp = std::string::npos;
    for (size_t i = pos; i < n; ++i) {
      if (text[i] == '!') {
        while (i < n && text[i] != '\n') ++i;
        continue;
      }
      if (text[i] == '&') { amp = i; break; }
    }
    if (amp == std::string::npos) break;
    size_t j = amp + 1;
    while (j < n && (std::isalnum((unsigned char)text[j]) || text[j] == '_')) ++j;
    std::string gname = lower(text.substr(amp + 1, j - amp - 1));
    if (gname == "end") { pos = j; continue; }
    std::string g = gname;
    if (g.size() > 4 && g.substr(g.size() - 4) == "_nml") g = g.substr(0, g.size() - 4);
    auto git = S.find(g);
    if (git == S.end()) {
      err = "unknown namelist group &" + gname;
      return false;
    }
    // body ends at '/' (outside strings/comments) or '&end'
    size_t k = j;
    bool in_str = false;
    char q = 0;
    size_t end = std::string::npos;
    for (; k < n; ++k) {
      char c = text[k];
      if (in_str) {
        if (c == q) in_str = false;
        continue;
      }
      if (c == '\'' || c == '"') { in_str = true; q = c; continue; }
      if (c == '!') {
        while (k < n && text[k] != '\n') ++k;
        continue;
      }
      if (c == '/') { end = k; break; }
      if (c == '&') { end = k; break; }
    }
    if (end == std::string::npos) {
      err = "namelist group &" + gname + " is not terminated by '/'";
      return false;
    }
    std::string body = text.substr(j, end - j);
    pos = (text[end] == '/') ? end + 1 : end;
    if (text[end] == '&') {
      // "&end" terminator
      size_t e2 = end + 1;
      while (e2 < n && std::isalpha((unsigned char)text[e2])) ++e2;
      if (lower(text.substr(end + 1, e2 - end - 1)) == "end") pos = e2;
    }
    std::vector<Tok> toks;
    if (!tokenize(body, toks, err)) {
      err = "&" + gname + ": " + err;
      return false;
    }
    size_t t = 0;
    while (t < toks.size()) {
      if (toks[t].kind == Tok::kComma) { ++t; continue; }
      if (toks[t].kind != Tok::kName) {
        err = "&" + gname + ": expected a key name, got '" + toks[t].text + "'";
        return false;
      }
      std::string key = lower(toks[t].text);
      ++t;
      int index = 0;
      if (t < toks.size() && toks[t].kind == Tok::kLParen) {
        if (t + 2 >= toks.size() || toks[t + 2].kind != Tok::kRParen ||
            !parse_int(toks[t + 1].text, index) || index < 1) {
          err = "&" + gname + ": bad array index for '" + key + "'";
          return false;
        }
        index -= 1;
        t += 3;
      }
      if (t >= toks.size() || toks[t].kind != Tok::kEq) {
        err = "&" + gname + ": expected '=' after '" + key + "'";
        return false;
      }
      ++t;
      std::vector<std::string> vals;
      std::vector<bool> quoted;
      while (t < toks.size() && toks[t].kind != Tok::kName) {
        if (toks[t].kind == Tok::kValue) {
          vals.push_back(toks[t].text);
          quoted.push_back(toks[t].quoted);
        }
        ++t;
      }
      expand_repeat(vals, quoted);
      auto kit = git->second.find(key);
      if (kit == git->second.end()) {
        err = "&" + gname + ": unknown key '" + key + "'";
        return false;
      }
      if (!check_value(kit->second.kind, vals, quoted)) {
        err = "&" + gname + ": invalid value for '" + key + "'";
        return false;
      }
      if (kit->second.set) kit->second.set(cfg, vals, index);
    }
  }
  return true;
}

int bc_code(const std::string& name) {
  static const std::map<std::string, int> m = {
      {"wall", 1}, {"open", 2}, {"tidal", 3}, {"nested", 4}, {"inflow", 5},
      {"discharge", 6}, {"clamped", 7}, {"sponge", 8}, {"chapman", 9}};
  auto it = m.find(trim(name));
  return it == m.end() ? 1 : it->second;
}

int scheme_code(const std::string& name) {
  std::string s = trim(name);
  if (s == "euler") return 1;
  if (s == "rk3") return 3;
  if (s == "rk43") return 4;
  return 2;
}

int validate(Config& c, std::string& err) {
  auto in = [](const std::string& v, std::initializer_list<const char*> allowed) {
    for (auto a : allowed)
      if (v == a) return true;
    return false;
  };
  // apply_time_unit_cascade (rki_config.F90:780-812)
  const std::string tu = trim(c.time_unit);
  double factor;
  if (in(tu, {"s", "sec", "second", "seconds"})) factor = 1.0;
  else if (in(tu, {"min", "minute", "minutes"})) factor = 60.0;
  else if (in(tu, {"hr", "hour", "hours", "h"})) factor = 3600.0;
  else if (in(tu, {"day", "days", "d"})) factor = 86400.0;
  else if (in(tu, {"year", "years", "yr"})) factor = 365.25 * 86400.0;
  else { err = "invalid time_unit '" + tu + "'"; return -2; }
  c.t_end = c.t_end * factor;

  if (c.sim_type != "coastal") { err = "sim_type must be 'coastal'"; return -2; }
  if (!in(c.grid_type, {"structured", "unstructured"})) { err = "invalid grid_type"; return -2; }
  if (c.nx < 1 || c.ny < 1) { err = "nx and ny must be >= 1"; return -2; }
  if (c.nghost < 1) { err = "nghost must be >= 1"; return -2; }
  if (!(c.dx > 0.0) || !(c.dy > 0.0)) { err = "dx and dy must be > 0"; return -2; }
  if (!(c.cfl > 0.0) || c.cfl > 1.0) { err = "cfl must be in (0, 1]"; return -2; }
  if (!(c.t_end > 0.0)) { err = "t_end must be > 0"; return -2; }
  if (c.cfl_interval < 1) { err = "cfl_interval must be >= 1"; return -2; }
  if (c.sponge_width < 0) { err = "sponge_width must be >= 0"; return -2; }
  if (c.n_tidal_constituents < 0 || c.n_tidal_constituents > kMaxTidalCfg) {
    err = "n_tidal_constituents must be in [0, 10]"; return -2;
  }
  if (!in(c.time_scheme, {"euler", "rk2", "rk3", "rk43", "semi_implicit"})) {
    err = "invalid time_scheme '" + c.time_scheme + "'"; return -2;
  }
  for (const std::string* b : {&c.bc_west, &c.bc_east, &c.bc_south, &c.bc_north})
    if (!in(*b, {"wall", "open", "tidal", "nested", "inflow", "discharge", "clamped", "sponge",
                 "chapman"})) {
      err = "invalid boundary type '" + *b + "'"; return -2;
    }
  if (!in(c.init_condition, {"dam_break", "gaussian_hump", "castro_dam_break", "still_water"})) {
    err = "invalid init_condition '" + c.init_condition + "'"; return -2;
  }
  if (!in(c.log_level, {"debug", "verbose", "info", "performance", "warning", "error"})) {
    err = "invalid log_level '" + c.log_level + "'"; return -2;
  }
  // The flux stencil reads two cells beyond the interior (rki_kernel_flux.F90:148-156).
  if (c.nghost < 2) { err = "nghost must be >= 2 for the 5-point flux stencil"; return -2; }
  // Solver modes outside the structured 2D barotropic step.
  if (c.grid_type != "structured") { err = "grid_type='unstructured' is not provided"; return -3; }
  if (c.use_multilayer) { err = "use_multilayer is not provided (2D barotropic only)"; return -3; }
  if (c.use_nonhydrostatic) { err = "use_nonhydrostatic is not provided"; return -3; }
  if (c.time_scheme == "semi_implicit") { err = "time_scheme='semi_implicit' is unstructured-only"; return -3; }
  return 0;
}

}  // namespace rkb
