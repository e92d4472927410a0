// bin/esp for thorx: runs THOR's large step from a .thr configuration file, in C++ over the C ABI
// of libthorx (include/thorx.h).
//
//     esp [config.thr] [-g GPU] [-o DIR] [-N STEPS] [-i FILE | -c FILE | -b] [-w]
//
// The program entry of the reference (src/esp.cu:164-1573): the same command-line arguments with
// the same meaning (src/esp.cu:183-198, overrides at :497-570), the same configuration syntax
// (key = value lines, comments, typed values; src/utils/config_file.cpp:60-130,
// src/headers/parser_helpers.h:77-365), the same keys and defaults for everything on the path
// (src/esp.cu:257-475, src/headers/define.h; the RT module's keys,
// src/physics/modules/src/radiative_transfer.cu:1107-1190; the insolation keys,
// src/ESP/insolation.cu:239-251), the same checks (src/esp.cu:574-700), the main loop's cadence
// of outputs, global diagnostics and log lines (src/esp.cu:1381-1480), batch and continue modes
// (src/esp.cu:848-940) and the three text logs (src/utils/log_writer.cpp). Output files are HDF5
// in the reference's layout (src/ESP/esp_output.cu:136-487), written by h5file.cpp.
//
// Differences, each where it applies: the grid file lacks the curl operator (not built) and the
// state files the RT's Qheat scaling; keys for physics this build does not implement are accepted
// at their default values and rejected with an error naming the key otherwise; output_mean,
// out_interm_momentum and output_diffusion are accepted with a warning that the arrays are not
// written; one extension key, `precision` = fp64 | mixed, selects the compute form. Restarts read
// HDF5 files only. Options beyond the reference's, for checking this program without a GPU:
// --dump-config prints the parsed and checked configuration and exits; --h5-dump FILE prints
// the datasets of an HDF5 file; --h5-copy IN OUT rewrites the datasets of IN into OUT with this
// program's writer.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <charconv>
#include <chrono>
#include <csignal>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <map>
#include <memory>
#include <regex>
#include <sstream>
#include <string>
#include <vector>

#include "thorx.h"
#include "h5file.h"

namespace fs = std::filesystem;

namespace {

constexpr double kAU    = 149597870700.0; // src/headers/physical_constants.h:9
constexpr double kRSun  = 695700000.0;    // src/headers/physical_constants.h:15
constexpr int    kError = 255;            // the reference's exit status on errors

void say(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vfprintf(stdout, fmt, ap);
    va_end(ap);
    std::fflush(stdout);
}

// ---------------------------------------------------------------------------------------------
// Configuration values and keys
// ---------------------------------------------------------------------------------------------
enum class Kind { Bool, Int, Double, String };
enum class Role { Path, Output, Fixed, Ignored }; // as thor_b200/esp.py: used, output only,
                                                  // must keep an allowed value, no effect here
struct Value {
    Kind        kind;
    bool        b = false;
    long long   i = 0;
    double      d = 0.0;
    std::string s;
};
Value B(bool v) { Value x{Kind::Bool}; x.b = v; return x; }
Value I(long long v) { Value x{Kind::Int}; x.i = v; return x; }
Value D(double v) { Value x{Kind::Double}; x.d = v; return x; }
Value S(const char* v) { Value x{Kind::String}; x.s = v; return x; }

// Python's repr of a float (shortest round-trip digits; exponent form below 1e-4 and from 1e16),
// so that messages read as the Python runner's
std::string py_float(double v) {
    if (v == 0.0)
        return std::signbit(v) ? "-0.0" : "0.0";
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
    std::string s(buf, r.ptr);
    const bool  neg = s[0] == '-';
    if (neg)
        s.erase(0, 1);
    const size_t e = s.find('e');
    const int    E = std::atoi(s.c_str() + e + 1);
    std::string  digits;
    for (size_t k = 0; k < e; k++)
        if (s[k] != '.')
            digits += s[k];
    const int   decpt = E + 1;
    std::string out;
    if (decpt <= -4 || decpt > 16) {
        out = digits.substr(0, 1);
        if (digits.size() > 1)
            out += "." + digits.substr(1);
        char eb[16];
        std::snprintf(eb, sizeof eb, "e%c%02d", E < 0 ? '-' : '+', std::abs(E));
        out += eb;
    }
    else if (decpt <= 0)
        out = "0." + std::string(-decpt, '0') + digits;
    else if ((int)digits.size() <= decpt)
        out = digits + std::string(decpt - digits.size(), '0') + ".0";
    else
        out = digits.substr(0, decpt) + "." + digits.substr(decpt);
    return (neg ? "-" : "") + out;
}
std::string py_str(const Value& v) {
    switch (v.kind) {
    case Kind::Bool: return v.b ? "True" : "False";
    case Kind::Int: return std::to_string(v.i);
    case Kind::Double: return py_float(v.d);
    default: return v.s;
    }
}
bool same(const Value& a, const Value& b) {
    if (a.kind != b.kind)
        return false;
    switch (a.kind) {
    case Kind::Bool: return a.b == b.b;
    case Kind::Int: return a.i == b.i;
    case Kind::Double: return a.d == b.d;
    default: return a.s == b.s;
    }
}

struct Key {
    const char* name;
    Value       def;
    Role        role;
};
// Defaults as the reference registers them: the planet's from SimulationSetup
// (src/ESP/simulation_setup.cu:60-76, a hot Jupiter), the switches from src/headers/define.h, and
// its own choice for MetStar, Tstar, radius_star and planet_star_dist, which take the defaults of
// Tint, kappa_lw, kappa_sw and f_lw (src/esp.cu:426-430).
const std::vector<Key>& keys() {
    static const std::vector<Key> k = {
        {"config_version", I(-1), Role::Ignored},
        {"timestep", I(1800), Role::Path},
        {"num_steps", I(48000), Role::Path},
        {"simulation_ID", S("Earth"), Role::Path},
        {"radius", D(72427000.0), Role::Path},
        {"rotation_rate", D(9.09e-5), Role::Path},
        {"gravitation", D(47.0), Role::Path},
        {"GravHeightVar", B(false), Role::Path},
        {"Rd", D(3714.0), Role::Path},
        {"Cp", D(13000.0), Role::Path},
        {"Tmean", D(1400.0), Role::Path},
        {"P_ref", D(10000000.0), Role::Path},
        {"Top_altitude", D(1235376.0), Role::Path},
        {"Diffc", D(0.009973), Role::Path},
        {"DivDampc", D(0.009973), Role::Path},
        {"Diffc_v", D(0.0), Role::Path},
        {"spring_dynamics", B(true), Role::Path},
        {"glevel", I(4), Role::Path},
        {"spring_beta", D(1.15), Role::Path},
        {"vlevel", I(32), Role::Path},
        {"HyDiff", B(true), Role::Path},
        {"HyDiffOrder", I(4), Role::Path},
        {"DivDampP", B(true), Role::Path},
        {"VertHyDiff", B(false), Role::Path},
        {"VertHyDiffOrder", I(6), Role::Path},
        {"increased_damping_for_n_steps", I(0), Role::Fixed},
        {"NonHydro", B(true), Role::Path},
        {"DeepModel", B(true), Role::Path},
        {"output_mean", B(true), Role::Output},
        {"out_interm_momentum", B(false), Role::Output},
        {"output_diffusion", B(false), Role::Output},
        {"RayleighSponge", B(false), Role::Path},
        {"RayleighSpongeT", B(false), Role::Path},
        {"DiffSponge", B(false), Role::Fixed},
        {"shrink_sponge", B(false), Role::Path},
        {"t_shrink", I(144000), Role::Path},
        {"raysp_calc_mode", S("imp"), Role::Path},
        {"nlat_bins", I(20), Role::Path},
        {"Ruv_sponge", D(1e-4), Role::Path},
        {"Rw_sponge", D(1e-4), Role::Path},
        {"RT_sponge", D(1e-4), Role::Path},
        {"ns_ray_sponge", D(0.75), Role::Path},
        {"damp_uv_to_mean", B(true), Role::Path},
        {"damp_w_to_mean", B(true), Role::Path},
        {"Dv_sponge", D(0.01), Role::Ignored},
        {"ns_diff_sponge", D(0.75), Role::Ignored},
        {"order_diff_sponge", I(2), Role::Ignored},
        {"rest", B(true), Role::Path},
        {"initial", S("ifile/esp_initial.h5"), Role::Path},
        {"core_benchmark", S("HeldSuarez"), Role::Path},
        {"init_PT_profile", S("isothermal"), Role::Fixed},
        {"conv_adj", B(false), Role::Path},
        {"conv_adj_iter", I(1), Role::Path},
        {"soft_adjustment", B(false), Role::Path},
        {"conv_adj_type", S("hourdin"), Role::Fixed},
        {"GPU_ID_N", I(0), Role::Path},
        {"n_out", I(1000), Role::Path},
        {"results_path", S("results"), Role::Path},
        {"gcm_off", B(false), Role::Path},
        {"globdiag", B(false), Role::Path},
        {"single_column", B(false), Role::Fixed},
        {"custom_global_n_out", B(false), Role::Path},
        {"global_n_out", I(1000), Role::Path},
        {"custom_log_n_out", B(false), Role::Path},
        {"log_n_out", I(1000), Role::Path},
        {"Tint", D(100.0), Role::Path},
        {"kappa_lw", D(0.002), Role::Path},
        {"kappa_sw", D(0.001), Role::Path},
        {"f_lw", D(0.5), Role::Path},
        {"bv_freq", D(0.01), Role::Ignored},
        {"MetStar", D(100.0), Role::Ignored},
        {"Tstar", D(0.002), Role::Path},
        {"radius_star", D(0.001), Role::Path},
        {"planet_star_dist", D(0.5), Role::Path},
        {"ultrahot_thermo", S("none"), Role::Fixed},
        {"ultrahot_heating", S("none"), Role::Fixed},
        {"thermo_equation", S("entropy"), Role::Path},
        {"vert_refined", B(false), Role::Fixed},
        {"transition_altitude", D(1000.0), Role::Ignored},
        {"lowest_layer_thickness", D(2.0), Role::Ignored},
        {"vert_dense_around", B(false), Role::Fixed},
        {"frac_height_dense", D(0.7), Role::Ignored},
        {"a_dense", D(1.0), Role::Ignored},
        {"b_dense", D(6.0), Role::Ignored},
        // physics modules (src/physics/managers/multi/src/phy_modules.cu:118-140)
        {"radiative_transfer", B(false), Role::Path},
        {"chemistry", B(false), Role::Fixed},
        {"chem_time_file", S(""), Role::Ignored},
        {"chem_fEQ_file", S(""), Role::Ignored},
        {"boundary_layer", B(false), Role::Fixed},
        {"bl_type", S("RayleighHS"), Role::Ignored},
        {"two_streams_radiative_transfer", B(false), Role::Fixed},
        // double-gray RT (radiative_transfer.cu:1146-1190, radiative_transfer.h:98-119)
        {"rt_type", S("DualbandGray"), Role::Fixed},
        {"diff_ang", D(0.5), Role::Path},
        {"albedo", D(0.18), Role::Path},
        {"latf_lw", B(false), Role::Path},
        {"kappa_lw_pole", D(0.002), Role::Path},
        {"n_sw", D(1.0), Role::Path},
        {"n_lw", D(2.0), Role::Path},
        {"rt1Dmode", B(false), Role::Path},
        {"surface", B(false), Role::Fixed},
        {"Csurf", D(1e7), Role::Ignored},
        {"dgrt_spinup_start", I(-1), Role::Path},
        {"dgrt_spinup_stop", I(-1), Role::Path},
        {"dgrt_spindown_start", I(-1), Role::Path},
        {"dgrt_spindown_stop", I(-1), Role::Path},
        // insolation (src/ESP/insolation.cu:239-251, src/headers/insolation.h:132-138)
        {"sync_rot", B(true), Role::Path},
        {"mean_motion", D(1.991e-7), Role::Path},
        {"alpha_i", D(0.0), Role::Path},
        {"true_long_i", D(0.0), Role::Path},
        {"ecc", D(0.0), Role::Path},
        {"obliquity", D(0.0), Role::Path},
        {"longp", D(0.0), Role::Path},
        {"insol_avg", S("NoInsolAvg"), Role::Fixed},
        // extension: compute form of this build
        {"precision", S("fp64"), Role::Path},
    };
    return k;
}
// values a Fixed key may take (its default unless listed)
const std::map<std::string, std::vector<Value>>& allowed() {
    static const std::map<std::string, std::vector<Value>> a = {
        {"init_PT_profile", {S("isothermal"), S("guillot")}},
        {"rt_type", {S("DualbandGray")}},
        {"conv_adj_type", {S("hourdin"), S("Hourdin")}},
        {"ultrahot_thermo", {S("none")}},
        {"ultrahot_heating", {S("none")}},
        {"insol_avg", {S("NoInsolAvg")}},
    };
    return a;
}
const std::vector<std::pair<std::string, std::vector<std::string>>>& choices() {
    static const std::vector<std::pair<std::string, std::vector<std::string>>> c = {
        {"core_benchmark", {"HeldSuarez", "NoBenchmark", "TidallyLockedEarth", "ShallowHotJupiter"}},
        {"thermo_equation", {"entropy", "energy"}},
        {"precision", {"fp64", "mixed"}},
    };
    return c;
}

struct Config {
    std::map<std::string, Value> v;
    bool        b(const char* k) const { return v.at(k).b; }
    long long   i(const char* k) const { return v.at(k).i; }
    double      d(const char* k) const { return v.at(k).d; }
    std::string s(const char* k) const { return v.at(k).s; }
};

// ---------------------------------------------------------------------------------------------
// Configuration syntax (src/headers/parser_helpers.h:77-130, 268-360)
// ---------------------------------------------------------------------------------------------
const char* kPunct = "!\"#$%&'()*+,\\-./:;<=>?@\\[\\\\\\]^_`{|}~";

bool parse_value(Kind kind, const std::string& text, Value& out) {
    static const std::regex re_bool("^(true|false)$");
    static const std::regex re_int("^((-|\\+)?[0-9]+)$");
    static const std::regex re_double("^((-|\\+)?[0-9]+(\\.[0-9]+)?((E|e)(-|\\+)?[0-9]+)?)$");
    out.kind = kind;
    switch (kind) {
    case Kind::Bool:
        if (!std::regex_match(text, re_bool))
            return false;
        out.b = text == "true";
        return true;
    case Kind::Int:
        if (!std::regex_match(text, re_int))
            return false;
        errno = 0;
        out.i = std::strtoll(text.c_str(), nullptr, 10);
        return errno == 0;
    case Kind::Double:
        if (!std::regex_match(text, re_double))
            return false;
        out.d = std::strtod(text.c_str(), nullptr);
        return true;
    default:
        out.s = text;
        return true;
    }
}

// Python's str.splitlines on the separators an ASCII file can hold
std::vector<std::string> split_lines(const std::string& t) {
    std::vector<std::string> out;
    std::string              cur;
    for (size_t k = 0; k < t.size(); k++) {
        const char ch = t[k];
        if (ch == '\n' || ch == '\r' || ch == '\v' || ch == '\f' || ch == '\x1c' || ch == '\x1d'
            || ch == '\x1e') {
            if (ch == '\r' && k + 1 < t.size() && t[k + 1] == '\n')
                k++;
            out.push_back(cur);
            cur.clear();
        }
        else
            cur += ch;
    }
    if (!cur.empty())
        out.push_back(cur);
    return out;
}

// Parses a .thr text into values with defaults, as the reference's config_file does: unknown
// keys warn and are skipped, a malformed line or value fails the whole file.
bool read_config(const std::string& text, Config& c) {
    for (const Key& k : keys())
        c.v[k.name] = k.def;
    static const std::regex re_empty("^[ \\t]*$");
    static const std::regex re_comment("^[ \\t]?#.*$");
    static const std::regex re_kv(std::string("^[ \\t]*([A-Za-z0-9_]+)[ \\t]*=[ \\t]*((?:[A-Za-z0-9]|[")
                                  + kPunct + "])+)[ \\t]*(#.*)?$");
    bool ok = true;
    int  n  = 0;
    for (const std::string& line : split_lines(text)) {
        n++;
        if (std::regex_match(line, re_empty) || std::regex_match(line, re_comment))
            continue;
        std::smatch m;
        if (!std::regex_match(line, m, re_kv)) {
            say("ERROR in config file at line %d :\t [%s]\n", n, line.c_str());
            ok = false;
            continue;
        }
        const std::string key = m[1], value = m[2];
        auto              it = c.v.find(key);
        if (it == c.v.end()) {
            say("WARNING: config file key [%s] does not exist, skipping\n", key.c_str());
            continue;
        }
        Value parsed;
        if (!parse_value(it->second.kind, value, parsed)) {
            say("ERROR: parsing of value [%s] failed for key [%s] \n", value.c_str(), key.c_str());
            ok = false;
            continue;
        }
        it->second = parsed;
    }
    return ok;
}

// The reference's range checks (src/esp.cu:574-700) plus this build's scope; prints every
// problem and returns false if there is one.
bool check_config(const Config& c) {
    std::vector<std::string> bad;
    auto need = [&](bool cond, const std::string& msg) {
        if (!cond)
            bad.push_back(msg);
    };
    need(c.i("timestep") > 0, "timestep must be > 0");
    need(c.i("num_steps") > 0, "nsmax must be > 0");
    need(c.d("gravitation") > 0, "gravitation must be > 0");
    need(c.d("Rd") > 0, "Rd must be > 0");
    need(c.d("Tmean") > 0, "T_mean must be > 0");
    need(c.d("P_ref") > 0, "P_Ref must be > 0");
    need(c.d("Top_altitude") > 0, "Top_altitude must be > 0");
    need(3 <= c.i("glevel") && c.i("glevel") <= 8, "glevel must be in [3, 8]");
    need(4 <= c.i("glevel") && c.i("glevel") <= 7,
         "glevel = " + std::to_string(c.i("glevel")) + ": this build's grid takes 4 to 7");
    need(c.i("vlevel") > 0, "vlevel must be > 0");
    need(c.i("GPU_ID_N") > -1, "GPU_ID_N must be > -1");
    need(c.i("n_out") > 0, "n_out must be > 0");
    need(c.s("simulation_ID").size() < 160, "Bad value for config variable simulation_ID");
    need(c.i("HyDiffOrder") > 2 && c.i("HyDiffOrder") % 2 == 0,
         "Bad value for HyDiffOrder! Must be multiple of 2 greater than/equal to 4.");
    need(c.i("VertHyDiffOrder") > 2 && c.i("VertHyDiffOrder") % 2 == 0,
         "Bad value for VertHyDiffOrder! Must be multiple of 2 greater than/equal to 4.");
    for (const auto& ch : choices()) {
        const std::string& v  = c.v.at(ch.first).s;
        bool               in = std::find(ch.second.begin(), ch.second.end(), v) != ch.second.end();
        std::string        list;
        for (size_t k = 0; k < ch.second.size(); k++)
            list += (k ? " | " : "") + ch.second[k];
        need(in, ch.first + " = " + v + ": this build supports " + list);
    }
    if (c.b("RayleighSponge")) { // src/esp.cu:757-780: the mode is read only with the sponge on
        const std::string m = c.s("raysp_calc_mode");
        need(m == "imp" || m == "exp1" || m == "exp3",
             "raysp_calc_mode config item not recognised: [" + m + "]");
        need(c.i("nlat_bins") >= 1, "nlat_bins must be >= 1");
        need(0.0 <= c.d("ns_ray_sponge") && c.d("ns_ray_sponge") < 1.0,
             "ns_ray_sponge must be in [0, 1)");
    }
    for (const Key& k : keys()) {
        if (k.role != Role::Fixed)
            continue;
        auto               it = allowed().find(k.name);
        std::vector<Value> ok = it != allowed().end() ? it->second : std::vector<Value>{k.def};
        bool               in = false;
        std::string        list;
        for (size_t j = 0; j < ok.size(); j++) {
            in = in || same(c.v.at(k.name), ok[j]);
            list += (j ? ", " : "") + py_str(ok[j]);
        }
        need(in, std::string(k.name) + " = " + py_str(c.v.at(k.name))
                     + ": not implemented in this build (allowed: " + list + ")");
    }
    if (!bad.empty()) {
        for (const auto& b : bad)
            say("Config error: %s\n", b.c_str());
        return false;
    }
    for (const char* k : {"output_mean", "out_interm_momentum", "output_diffusion"})
        if (c.b(k))
            say("WARNING: %s = true: those arrays are not written by this build\n", k);
    return true;
}

// ---------------------------------------------------------------------------------------------
// The configuration as the C ABI's parameter structs
// ---------------------------------------------------------------------------------------------
int benchmark_of(const std::string& s) {
    if (s == "NoBenchmark")
        return THORX_NO_BENCHMARK;
    if (s == "TidallyLockedEarth")
        return THORX_TIDALLY_LOCKED_EARTH;
    if (s == "ShallowHotJupiter")
        return THORX_SHALLOW_HOT_JUPITER;
    return THORX_HELD_SUAREZ;
}
thorx_params dycore_params(const Config& c) {
    thorx_params p{};
    p.A               = c.d("radius");
    p.Omega           = c.d("rotation_rate");
    p.Gravit          = c.d("gravitation");
    p.Rd              = c.d("Rd");
    p.Cp              = c.d("Cp");
    p.P_Ref           = c.d("P_ref");
    p.Top_altitude    = c.d("Top_altitude");
    p.timestep        = (double)c.i("timestep");
    p.Diffc           = c.d("Diffc");
    p.DivDampc        = c.d("DivDampc");
    p.HyDiffOrder     = (int)c.i("HyDiffOrder");
    p.DeepModel       = c.b("DeepModel");
    p.NonHydro        = c.b("NonHydro");
    p.GravHeightVar   = c.b("GravHeightVar");
    p.HyDiff          = c.b("HyDiff");
    p.DivDampP        = c.b("DivDampP");
    p.thermo_equation = c.s("thermo_equation") == "energy" ? THORX_ENERGY : THORX_ENTROPY;
    p.core_benchmark  = benchmark_of(c.s("core_benchmark"));
    p.precision       = c.s("precision") == "mixed" ? THORX_MIXED : THORX_FP64;
    return p;
}
thorx_sponge_params sponge_params(const Config& c, int first_step) {
    thorx_sponge_params s{};
    s.nlat_bins       = (int)c.i("nlat_bins");
    s.Ruv_sponge      = c.d("Ruv_sponge");
    s.Rw_sponge       = c.d("Rw_sponge");
    s.RT_sponge       = c.d("RT_sponge");
    s.ns_ray_sponge   = c.d("ns_ray_sponge");
    s.damp_uv_to_mean = c.b("damp_uv_to_mean");
    s.damp_w_to_mean  = c.b("damp_w_to_mean");
    s.RayleighSpongeT = c.b("RayleighSpongeT");
    s.shrink_sponge   = c.b("shrink_sponge");
    s.t_shrink        = (int)c.i("t_shrink");
    s.first_step      = first_step;
    const std::string m = c.s("raysp_calc_mode");
    s.raysp_calc_mode   = m == "exp1" ? 1 : m == "exp3" ? 2 : 0;
    return s;
}
// the RT module's parameters in the C ABI's units (m, K, degrees): the configuration gives the
// star radius in solar radii and the distance in au (src/ESP/esp_initial.cu:194-196)
thorx_rt_params rt_params(const Config& c, int first_step) {
    thorx_rt_params r{};
    r.Tstar            = c.d("Tstar");
    r.planet_star_dist = c.d("planet_star_dist") * kAU;
    r.radius_star      = c.d("radius_star") * kRSun;
    r.diff_ang         = c.d("diff_ang");
    r.Tint             = c.d("Tint");
    r.albedo           = c.d("albedo");
    r.kappa_sw         = c.d("kappa_sw");
    r.kappa_lw         = c.d("kappa_lw");
    r.kappa_lw_pole    = c.d("kappa_lw_pole");
    r.n_sw             = c.d("n_sw");
    r.n_lw             = c.d("n_lw");
    r.f_lw             = c.d("f_lw");
    r.mean_motion      = c.d("mean_motion");
    r.alpha_i          = c.d("alpha_i");
    r.true_long_i      = c.d("true_long_i");
    r.ecc              = c.d("ecc");
    r.obliquity        = c.d("obliquity");
    r.longp            = c.d("longp");
    r.latf_lw          = c.b("latf_lw");
    r.rt1Dmode         = c.b("rt1Dmode");
    r.sync_rot         = c.b("sync_rot");
    r.surface          = 0;
    r.spinup_start     = (int)c.i("dgrt_spinup_start");
    r.spinup_stop      = (int)c.i("dgrt_spinup_stop");
    r.spindown_start   = (int)c.i("dgrt_spindown_start");
    r.spindown_stop    = (int)c.i("dgrt_spindown_stop");
    r.first_step       = first_step;
    return r;
}

void dump_config(const Config& c) {
    for (const Key& k : keys())
        say("%s = %s\n", k.name, py_str(c.v.at(k.name)).c_str());
    const thorx_params p = dycore_params(c);
    say("# thorx_params: thermo_equation %d core_benchmark %d precision %d\n", p.thermo_equation,
        p.core_benchmark, p.precision);
    const thorx_rt_params r = rt_params(c, 1);
    say("# thorx_rt_params: planet_star_dist %s radius_star %s\n",
        py_float(r.planet_star_dist).c_str(), py_float(r.radius_star).c_str());
}

// ---------------------------------------------------------------------------------------------
// The simulation context
// ---------------------------------------------------------------------------------------------
struct Failure {
    std::string what;
};

class Sim {
  public:
    thorx_ctx* x = nullptr;
    ~Sim() {
        if (x)
            thorx_destroy(x);
    }
    void check(int rc, const char* call) const {
        if (rc != 0)
            throw Failure{std::string(call) + ": " + (x ? thorx_last_error(x) : "")};
    }
    long size(const char* name) const { return thorx_field_size(x, name); }
    std::vector<double> get(const char* name) const {
        const long n = size(name);
        if (n < 0)
            throw Failure{std::string("unknown field ") + name};
        std::vector<double> v((size_t)n);
        check(thorx_get_field(x, name, v.data()), "thorx_get_field");
        return v;
    }
    void set(const char* name, const std::vector<double>& v) {
        if ((long)v.size() != size(name))
            throw Failure{std::string(name) + ": size does not match"};
        check(thorx_set_field(x, name, v.data()), "thorx_set_field");
    }
};

struct Grid {
    thorx_icogrid* g = nullptr;
    ~Grid() {
        if (g)
            thorx_grid_free(g);
    }
    template<class T>
    std::vector<T> get(const char* name) const {
        const long     n = thorx_grid_get(g, name, nullptr);
        std::vector<T> v(n > 0 ? (size_t)n : 0);
        if (n > 0)
            thorx_grid_get(g, name, v.data());
        return v;
    }
};

// ---------------------------------------------------------------------------------------------
// Files: HDF5 outputs (src/ESP/esp_output.cu) and the text logs (src/utils/log_writer.cpp)
// ---------------------------------------------------------------------------------------------
std::string output_name(const std::string& sim_id, int idx) {
    return "esp_output_" + sim_id + "_" + std::to_string(idx) + ".h5";
}
std::string join(const std::string& dir, const std::string& name) {
    return (fs::path(dir) / name).string();
}
void table(thorx_h5::Writer& w, const char* name, const std::vector<double>& v, const char* unit,
           const char* desc) {
    w.table(name, v.data(), v.size(), unit, desc);
}
void finish(thorx_h5::Writer& w, const std::string& path) {
    std::string err;
    if (!w.close(path, &err))
        throw Failure{err};
}

// ESP::output's state file (src/ESP/esp_output.cu:306-470) and the RT module's and the
// insolation's store() (radiative_transfer.cu:1286-1336, insolation.cu:484-493)
void write_state(const std::string& path, const Sim& x, long long nstep, double sim_time,
                 const double* glob, const std::vector<std::vector<double>>* cells, bool rt) {
    thorx_h5::Writer w;
    w.value_i32("/nstep", (int32_t)nstep, "-", "Step number");
    w.value("/simulation_time", sim_time, "s", "Simulation time");
    table(w, "/Rho", x.get("Rho"), "kg/m^3", "Density");
    table(w, "/Pressure", x.get("pressure"), "Pa", "Pressure");
    table(w, "/Mh", x.get("Mh"), "kg m^-2 s^-1", "Horizontal Momentum");
    table(w, "/Wh", x.get("Wh"), "kg m^-2 s^-1", "Vertical Momentum");
    if (cells) { // the per-cell terms of the global sums (esp_output.cu:410-428)
        table(w, "/Etotal", (*cells)[0], "kg m^2/s^2", "Total Energy");
        table(w, "/Entropy", (*cells)[5], "kg m^2/s^2 K^-1", "Entropy");
        table(w, "/Mass", (*cells)[1], "kg", "Mass");
        table(w, "/AngMomx", (*cells)[2], "kg m^2/s", "AngMom in X");
        table(w, "/AngMomy", (*cells)[3], "kg m^2/s", "AngMom in Y");
        table(w, "/AngMomz", (*cells)[4], "kg m^2/s", "AngMom in Z");
    }
    if (glob) {
        w.value("/GlobalE", glob[0], "kg m^2/s^2", "Global Total Energy");
        w.value("/GlobalEnt", glob[5], "kg m^2/s^2 K^-1", "Global Entropy");
        w.value("/GlobalMass", glob[1], "kg", "Global Mass");
        w.value("/GlobalAMx", glob[2], "kg m^2/s", "Global AngMomX");
        w.value("/GlobalAMy", glob[3], "kg m^2/s", "Global AngMomY");
        w.value("/GlobalAMz", glob[4], "kg m^2/s", "Global AngMomZ");
    }
    table(w, "/Qheat", x.get("profx_Qheat"), "W m^-3", "Physics module Qheat");
    table(w, "/Rd", x.get("Rd"), "J/K/kg", "Local gas constant");
    table(w, "/Cp", x.get("Cp"), "J/K/kg", "Local heat capacity");
    if (rt) {
        double asr = 0, olr = 0;
        x.check(thorx_rt_totals(x.x, &asr, &olr), "thorx_rt_totals");
        table(w, "/insol", x.get("insol"), "W m^-2", "insolation (instantaneous)");
        table(w, "/insol_annual", x.get("insol_ann"), "W m^-2",
              "insolation (annual/orbit averaged)");
        table(w, "/flw_up", x.get("flw_up"), "W m^-2", "upward flux (LW)");
        table(w, "/fsw_up", x.get("fsw_up"), "W m^-2", "upward flux (SW)");
        table(w, "/flw_dn", x.get("flw_dn"), "W m^-2", "downward flux (LW)");
        table(w, "/fsw_dn", x.get("fsw_dn"), "W m^-2", "downward flux (SW)");
        table(w, "/tau", x.get("tau"), " ",
              "optical depth across each layer (not total optical depth)");
        table(w, "/DGQheat", x.get("DG_Qheat"), " ", "Double Gray Qheat");
        w.value("/ASR", asr, "W", "Absorbed Shortwave Radiation (global total)");
        w.value("/OLR", olr, "W", "Outgoing Longwave Radiation (global total)");
        table(w, "/cos_zenith_angles", x.get("cos_zenith"), "-", "cos_zenith_angles per column");
    }
    finish(w, path);
}

// ESP::output's grid file (src/ESP/esp_output.cu:144-183), without the curl operator
void write_grid(const std::string& path, const Grid& g, int point_num, int nv) {
    thorx_h5::Writer w;
    table(w, "/Altitude", g.get<double>("Altitude"), "m", "Altitude");
    table(w, "/Altitudeh", g.get<double>("Altitudeh"), "m", "Altitude at the interfaces");
    table(w, "/areasT", g.get<double>("areasT"), "m^2", "Main cells areas");
    table(w, "/lonlat", g.get<double>("lonlat"), "-", "Longitudes and latitudes");
    w.value("/point_num", (double)point_num, "-", "Number of grid points in one level");
    w.value("/nv", (double)nv, "-", "Number of vertical layers");
    const std::vector<int32_t> pl = g.get<int32_t>("point_local");
    w.table_i32("/pntloc", pl.data(), pl.size(), "-", "Neighbours indexes");
    table(w, "/grad", g.get<double>("grad"), "m^-1", "Horizontal gradient operator");
    table(w, "/div", g.get<double>("div"), "m^-1", "Horizontal divergence operator");
    finish(w, path);
}

// ESP::output's planet file (src/ESP/esp_output.cu:186-304) with the module manager's, the RT
// module's and the insolation's store_init (phy_modules.cu:219-237,
// radiative_transfer.cu:1366-1388, insolation.cu:459-479)
void write_planet(const std::string& path, const Config& c) {
    auto             b = [&](const char* k) { return c.b(k) ? 1.0 : 0.0; };
    thorx_h5::Writer w;
    w.value_i32("/glevel", (int32_t)c.i("glevel"), "-", "Horizontal subdivision level");
    w.value_i32("/vlevel", (int32_t)c.i("vlevel"), "-", "Vertical subdivision level");
    w.value("/spring_dynamics", b("spring_dynamics"), "-", "Spring dynamics");
    w.value("/spring_beta", c.d("spring_beta"), "-", "Spring Beta");
    w.value("/A", c.d("radius"), "m", "Planet radius");
    w.value("/Rd", c.d("Rd"), "J/(Kg K)", "Gas constant");
    w.value("/Omega", c.d("rotation_rate"), "1/s", "Rotation rate");
    w.value("/Gravit", c.d("gravitation"), "m/s^2", "Surface gravity");
    w.value("/P_Ref", c.d("P_ref"), "Pa", "Reference pressure");
    w.value("/Top_altitude", c.d("Top_altitude"), "m", "Top of the model's domain");
    w.value("/Cp", c.d("Cp"), "J/(Kg K)", "Specific heat capacity");
    w.value("/RayleighSponge", b("RayleighSponge"), "-", "Using Rayleigh SpongeLayer?");
    w.value("/RayleighSpongeT", b("RayleighSpongeT"), "-", "Using thermal SpongeLayer?");
    w.value("/DiffSponge", b("DiffSponge"), "-", "Using Diffusive SpongeLayer?");
    w.value("/DeepModel", b("DeepModel"), "-", "Using Deep Model");
    w.value("/NonHydro", b("NonHydro"), "-", "Using Non Hydrostatic parameter");
    w.value("/output_mean", b("output_mean"), "-", "outputting mean quantities");
    w.value("/output_diffusion", b("output_diffusion"), "-", "outputting diffusion terms");
    w.value("/out_interm_momentum", b("out_interm_momentum"), "-",
            "outputting intermediate momentum values");
    w.value("/DivDampP", b("DivDampP"), "-", "Using Divergence-damping");
    w.value("/HyDiff", b("HyDiff"), "-", "Using Hyper diffusion");
    w.value("/Diffc", c.d("Diffc"), "-", "Hyperdiffusion strength");
    w.value("/Diffc_v", c.d("Diffc_v"), "-", "Vertical hyperdiffusion strength");
    w.value("/Tmean", c.d("Tmean"), "K", "Mean atmospheric temperature");
    w.value("/conv_adj", b("conv_adj"), "-", "Using convection adjustment");
    w.value("/gcm_off", b("gcm_off"), "-", "GCM off");
    w.value("/single_column", b("single_column"), "-", "single column mode");
    w.value("/rest", b("rest"), "-", "Starting from rest");
    w.value_i32("/core_benchmark", benchmark_of(c.s("core_benchmark")), "-",
                "Using benchmark forcing");
    if (c.b("RayleighSponge")) {
        w.value_i32("/nlat_bins", (int32_t)c.i("nlat_bins"), "-",
                    "number of lat rings for Rayleigh sponge layer");
        w.value("/ns_ray_sponge", c.d("ns_ray_sponge"), "-", "Bottom of rayleigh sponge layer");
        w.value("/Ruv_sponge", c.d("Ruv_sponge"), "1/s",
                "Strength of Rayleigh sponge layer (uv components)");
        w.value("/Rw_sponge", c.d("Rw_sponge"), "1/s",
                "Strength of Rayleigh sponge layer (w component)");
    }
    w.value("/Tint", c.d("Tint"), "K", "Temperature of interior heat flux");
    w.value("/f_lw", c.d("f_lw"), "-", "fraction of taulw in well-mixed absorber");
    w.value("/kappa_lw", c.d("kappa_lw"), "-", "longwave opacity");
    w.value("/kappa_sw", c.d("kappa_sw"), "-", "shortwave opacity");
    w.value("/phy_module", 0.0, "-", "multi");
    w.value("/surface", 0.0, "-", "include solid/liquid surface");
    w.value("/Csurf", c.d("Csurf"), "J/K/m^2", "heat capacity of surface by area");
    // the module manager (multi) and its modules
    w.value("/radiative_transfer", b("radiative_transfer"), "-", "Using radiative transfer");
    w.value("/Tstar", c.d("Tstar"), "K", "Temperature of host star");
    w.value("/planet_star_dist", c.d("planet_star_dist"), "au", "distance b/w host star and planet");
    w.value("/radius_star", c.d("radius_star"), "R_sun", "radius of host star");
    w.value("/diff_ang", c.d("diff_ang"), "-", "diffusivity factor");
    w.value("/albedo", c.d("albedo"), "-", "bond albedo of planet");
    w.value("/latf_lw", b("latf_lw"), "-", "use lat dependent opacity");
    w.value("/kappa_lw_pole", c.d("kappa_lw_pole"), "-", "gray opacity of longwave at poles");
    w.value("/n_lw", c.d("n_lw"), "-", "power law exponent for unmixed absorber in LW");
    w.value("/n_sw", c.d("n_sw"), "-", "power law exponent for mixed/unmixed absorber in SW");
    w.value_i32("/rt_type", 0, "-", "Type of radiative transfer physics");
    w.value("/chemistry", 0.0, "-", "Using relaxation chemistry");
    w.value("/boundary_layer", 0.0, "-", "Using boundary layer");
    if (c.b("radiative_transfer")) {
        w.value("/sync_rot", b("sync_rot"), "-", "enforce synchronous rotation");
        w.value("/mean_motion", c.d("mean_motion"), "rad/s", "orbital mean motion");
        w.value("/alpha_i", c.d("alpha_i"), "deg", "initial RA of host star");
        w.value("/true_long_i", c.d("true_long_i"), "deg", "initial orbital position of planet");
        w.value("/ecc", c.d("ecc"), "-", "orbital eccentricity");
        w.value("/obliquity", c.d("obliquity"), "deg", "tilt of spin axis");
        w.value("/longp", c.d("longp"), "deg", "longitude of periastron");
    }
    finish(w, path);
}

// (basename, number) of a file named esp_output_<basename>_<number>.h5
// (match_output_file_numbering_scheme, src/utils/directories.cpp:270-311)
bool output_numbering(const std::string& path, std::string& base, int& number) {
    const std::string name = fs::path(path).filename().string();
    if (name.size() < 3 || name.compare(name.size() - 3, 3, ".h5") != 0)
        return false;
    std::vector<std::string> parts;
    std::stringstream        ss(name.substr(0, name.size() - 3));
    for (std::string p; std::getline(ss, p, '_');)
        parts.push_back(p);
    if (!name.empty() && name[name.size() - 4] == '_')
        parts.push_back("");
    if (parts.size() < 4 || parts[0] != "esp" || parts[1] != "output")
        return false;
    static const std::regex re_int("^[ \\t\\n]*[-+]?[0-9]+[ \\t\\n]*$");
    if (!std::regex_match(parts.back(), re_int))
        return false;
    number = std::atoi(parts.back().c_str());
    if (number <= -1)
        return false;
    base.clear();
    for (size_t k = 2; k + 1 < parts.size(); k++)
        base += (k > 2 ? "_" : "") + parts[k];
    return true;
}

// The planet file that goes with an initial-conditions file (find_continue_file,
// src/utils/directories.cpp:313-362); empty when continuing from a file without the output naming
std::string planet_file(const std::string& initial, bool continuing) {
    std::string dir = fs::path(initial).parent_path().string();
    if (dir.empty())
        dir = ".";
    std::string base;
    int         number;
    if (output_numbering(initial, base, number))
        return join(dir, "esp_output_planet_" + base + ".h5");
    if (continuing)
        return "";
    return join(dir, fs::path(initial).stem().string() + "_planet.h5");
}

// The restart check of src/ESP/esp_initial.cu:1147-1205: A, Top_altitude, glevel, vlevel and
// surface of the planet file must equal the configuration's
bool check_planet(const std::string& path, const Config& c) {
    std::map<std::string, thorx_h5::Dataset> d;
    std::string                              err;
    if (!thorx_h5::read(path, d, &err)) {
        say("planet_file %s not readable: %s\n", path.c_str(), err.c_str());
        return false;
    }
    struct Want {
        const char* key;
        double      v;
        bool        integer;
    };
    const Want want[] = {{"A", c.d("radius"), false},
                         {"Top_altitude", c.d("Top_altitude"), false},
                         {"glevel", (double)c.i("glevel"), true},
                         {"vlevel", (double)c.i("vlevel"), true},
                         {"surface", 0.0, false}};
    bool ok = true;
    for (const Want& wv : want) {
        auto it = d.find(wv.key);
        if (it == d.end() || it->second.values.empty()) {
            say("Error reading key /%s from reload config.\n", wv.key);
            ok = false;
            continue;
        }
        const double have = it->second.values[0];
        if (have != wv.v) {
            const std::string ws = wv.integer ? std::to_string((long long)wv.v) : py_float(wv.v);
            const std::string hs = it->second.integer ? std::to_string((long long)have)
                                                      : py_float(have);
            say("mismatch for /%s value between config value: %s and initial condition value "
                "%s.\n",
                wv.key, ws.c_str(), hs.c_str());
            ok = false;
        }
    }
    if (!ok)
        say("Could not reload full configuration.\n");
    return ok;
}

struct Start {
    std::map<std::string, std::vector<double>> fields; // the state the file holds
    long long                                  nstep = 0;
    double                                     time  = 0.0;
};
// what a restart reads (src/ESP/esp_initial.cu:1215-1260): the prognostic fields and the
// per-cell gas constants
bool read_state(const std::string& path, Start& st) {
    if (path.size() >= 4 && path.compare(path.size() - 4, 4, ".npz") == 0) {
        say("start file %s: .npz archives are not read by this program\n", path.c_str());
        return false;
    }
    std::map<std::string, thorx_h5::Dataset> d;
    std::string                              err;
    if (!thorx_h5::read(path, d, &err)) {
        say("start file %s not readable: %s\n", path.c_str(), err.c_str());
        return false;
    }
    const std::pair<const char*, const char*> names[] = {
        {"Rho", "Rho"}, {"pressure", "Pressure"}, {"Mh", "Mh"}, {"Wh", "Wh"}, {"Rd", "Rd"},
        {"Cp", "Cp"}};
    for (const auto& n : names)
        if (d.count(n.second))
            st.fields[n.first] = d[n.second].values;
    if (!d.count("nstep") || !d.count("simulation_time") || d["nstep"].values.empty()
        || d["simulation_time"].values.empty()) {
        say("start file %s lacks nstep or simulation_time\n", path.c_str());
        return false;
    }
    st.nstep = (long long)d["nstep"].values[0];
    st.time  = d["simulation_time"].values[0];
    return true;
}

std::string g16(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.16g", v);
    return b;
}

// esp_write_log_<ID>.txt, esp_global_<ID>.txt, esp_diagnostics_<ID>.txt in the output directory,
// with the reference's headers and columns
class Logs {
  public:
    Logs(const std::string& dir, const std::string& id, bool append, bool globdiag) {
        write_log_ = open(join(dir, "esp_write_log_" + id + ".txt"), append,
                          "#step_number\tfile_number\tfilename");
        if (globdiag)
            glob_ = open(join(dir, "esp_global_" + id + ".txt"), append,
                         "#current_step\tsimulation_time\tGlobalE_h\tGlobalMass_h\tGlobalAMx_h\t"
                         "GlobalAMy_h\tGlobalAMz_h\tGlobalEnt_h");
        diag_ = open(join(dir, "esp_diagnostics_" + id + ".txt"), append,
                     "#current_step\tsimulation_time\ttotal_bytes\tfree_bytes\telapsed_time\t"
                     "time_left\tmean_delta_per_step\tend_time");
    }
    ~Logs() {
        for (FILE* f : {write_log_, glob_, diag_})
            if (f)
                std::fclose(f);
    }
    void output(long long step, int idx, const std::string& name) {
        std::fprintf(write_log_, "%lld\t%d\t%s\n", step, idx, name.c_str());
        std::fflush(write_log_);
    }
    void globdiag(long long step, double t, const double* g) {
        std::fprintf(glob_, "%lld\t%s", step, g16(t).c_str());
        for (int k = 0; k < 6; k++)
            std::fprintf(glob_, "\t%s", g16(g[k]).c_str());
        std::fprintf(glob_, "\n");
        std::fflush(glob_);
    }
    void diagnostics(long long step, double t, double elapsed, double left, double mean,
                     const std::string& end) {
        std::fprintf(diag_, "%lld\t%s\t%d\t%d\t%s\t%s\t%s\t%s\n", step, g16(t).c_str(), 0, 0,
                     g16(elapsed).c_str(), g16(left).c_str(), g16(mean).c_str(), end.c_str());
        std::fflush(diag_);
    }

  private:
    static FILE* open(const std::string& path, bool append, const char* header) {
        const bool fresh = !append || !fs::exists(path);
        FILE*      f     = std::fopen(path.c_str(), append ? "a" : "w");
        if (!f)
            throw Failure{"cannot open " + path};
        if (fresh)
            std::fprintf(f, "%s\n", header);
        return f;
    }
    FILE *write_log_ = nullptr, *glob_ = nullptr, *diag_ = nullptr;
};

// (file number, step, filename) of the last line of esp_write_log_<ID>.txt
// (log_writer::check_output_log, src/utils/log_writer.cpp:80-136)
bool last_output(const std::string& dir, const std::string& id, int& idx, long long& step,
                 std::string& name) {
    std::ifstream f(join(dir, "esp_write_log_" + id + ".txt"));
    if (!f)
        return false;
    bool found = false;
    for (std::string line; std::getline(f, line);) {
        if (line.empty() || line[0] == '#')
            continue;
        std::istringstream ss(line);
        std::string        a, b, c, extra;
        if (ss >> a >> b >> c && !(ss >> extra)) {
            step  = std::atoll(a.c_str());
            idx   = std::atoi(b.c_str());
            name  = c;
            found = true;
        }
    }
    return found;
}

// ---------------------------------------------------------------------------------------------
// Command line (src/esp.cu:183-198)
// ---------------------------------------------------------------------------------------------
struct Args {
    std::string config = "ifile/earth.thr";
    bool        has_gpu = false, has_out = false, has_init = false, has_cont = false;
    bool        has_steps = false, overwrite = false, batch = false, dump = false;
    int         gpu = 0;
    long long   steps = 0;
    std::string out, initial, cont, h5dump, h5copy_in, h5copy_out;
};
const char* kUsage =
    "usage: esp [-h] [-g GPU_ID] [-o OUTPUT_DIR] [-i INITIAL] [-c CONT] [-N NUMSTEPS] [-w] [-b]\n"
    "           [--dump-config] [--h5-dump FILE] [--h5-copy IN OUT] [config]\n";

// 0: parsed; 1: help printed; 2: usage error (printed)
int parse_args(int argc, char** argv, Args& a) {
    bool have_config = false;
    auto integer     = [](const std::string& s, long long& v) {
        static const std::regex re("^[ \\t]*[-+]?[0-9]+[ \\t]*$");
        if (!std::regex_match(s, re))
            return false;
        v = std::atoll(s.c_str());
        return true;
    };
    for (int k = 1; k < argc; k++) {
        std::string arg = argv[k], name, val;
        bool        attached = false;
        if (arg.size() > 2 && arg[0] == '-' && arg[1] == '-') {
            const size_t eq = arg.find('=');
            name            = arg.substr(0, eq);
            if (eq != std::string::npos)
                val = arg.substr(eq + 1), attached = true;
        }
        else if (arg.size() >= 2 && arg[0] == '-' && arg != "-") {
            name = arg.substr(0, 2);
            if (arg.size() > 2)
                val = arg.substr(2), attached = true;
        }
        else {
            if (have_config) {
                std::fprintf(stderr, "%sesp: error: unrecognized arguments: %s\n", kUsage,
                             arg.c_str());
                return 2;
            }
            a.config    = arg;
            have_config = true;
            continue;
        }
        auto value = [&](std::string& out) {
            if (!attached) {
                if (k + 1 >= argc) {
                    std::fprintf(stderr, "%sesp: error: argument %s: expected one argument\n",
                                 kUsage, name.c_str());
                    return false;
                }
                out = argv[++k];
            }
            else
                out = val;
            return true;
        };
        if (name == "-h" || name == "--help") {
            std::printf("%s", kUsage);
            return 1;
        }
        else if (name == "-w" || name == "--overwrite")
            a.overwrite = true;
        else if (name == "-b" || name == "--batch")
            a.batch = true;
        else if (name == "--dump-config")
            a.dump = true;
        else if (name == "-g" || name == "--gpu_id" || name == "-N" || name == "--numsteps") {
            std::string s;
            long long   v;
            if (!value(s))
                return 2;
            if (!integer(s, v)) {
                std::fprintf(stderr, "%sesp: error: argument %s: invalid int value: '%s'\n",
                             kUsage, name.c_str(), s.c_str());
                return 2;
            }
            if (name == "-g" || name == "--gpu_id")
                a.gpu = (int)v, a.has_gpu = true;
            else
                a.steps = v, a.has_steps = true;
        }
        else if (name == "-o" || name == "--output_dir") {
            if (!value(a.out))
                return 2;
            a.has_out = true;
        }
        else if (name == "-i" || name == "--initial") {
            if (!value(a.initial))
                return 2;
            a.has_init = true;
        }
        else if (name == "-c" || name == "--continue") {
            if (!value(a.cont))
                return 2;
            a.has_cont = true;
        }
        else if (name == "--h5-dump") {
            if (!value(a.h5dump))
                return 2;
        }
        else if (name == "--h5-copy") {
            if (!value(a.h5copy_in))
                return 2;
            if (k + 1 >= argc) {
                std::fprintf(stderr, "%sesp: error: argument --h5-copy: expected 2 arguments\n",
                             kUsage);
                return 2;
            }
            a.h5copy_out = argv[++k];
        }
        else {
            std::fprintf(stderr, "%sesp: error: unrecognized arguments: %s\n", kUsage, arg.c_str());
            return 2;
        }
    }
    return 0;
}

int h5_dump(const std::string& path) {
    std::map<std::string, thorx_h5::Dataset> d;
    std::string                              err;
    if (!thorx_h5::read(path, d, &err)) {
        say("%s\n", err.c_str());
        return kError;
    }
    for (const auto& kv : d) {
        const thorx_h5::Dataset& ds = kv.second;
        double                   sum = 0.0;
        for (double v : ds.values)
            sum += v;
        say("%s\t%s\t%zu\t%s\t%s\t%s\t%s\n", kv.first.c_str(), ds.integer ? "int" : "float",
            ds.values.size(), ds.attrs.count("units") ? ds.attrs.at("units").c_str() : "",
            ds.attrs.count("Variable") ? ds.attrs.at("Variable").c_str() : "",
            ds.values.empty() ? "" : g16(ds.values[0]).c_str(), g16(sum).c_str());
    }
    return 0;
}

int h5_copy(const std::string& in, const std::string& out) {
    std::map<std::string, thorx_h5::Dataset> d;
    std::string                              err;
    if (!thorx_h5::read(in, d, &err)) {
        say("%s\n", err.c_str());
        return kError;
    }
    thorx_h5::Writer w;
    for (const auto& kv : d) {
        const thorx_h5::Dataset& ds   = kv.second;
        auto                     attr = [&](const char* k) {
            return ds.attrs.count(k) ? ds.attrs.at(k) : std::string();
        };
        if (ds.integer) {
            std::vector<int32_t> v(ds.values.begin(), ds.values.end());
            w.table_i32(kv.first, v.data(), v.size(), attr("units"), attr("Variable"));
        }
        else
            w.table(kv.first, ds.values.data(), ds.values.size(), attr("units"), attr("Variable"));
    }
    if (!w.close(out, &err)) {
        say("%s\n", err.c_str());
        return kError;
    }
    return 0;
}

std::atomic<int> g_caught{0};
extern "C" void on_signal(int signum) { g_caught.store(signum); } // src/esp.cu:99-110

// ---------------------------------------------------------------------------------------------
// The run
// ---------------------------------------------------------------------------------------------
int run(int argc, char** argv) {
    Args a;
    if (int rc = parse_args(argc, argv, a))
        return rc == 1 ? 0 : 2;
    if (!a.h5dump.empty())
        return h5_dump(a.h5dump);
    if (!a.h5copy_in.empty())
        return h5_copy(a.h5copy_in, a.h5copy_out);
    std::string text;
    {
        std::ifstream f(a.config, std::ios::binary);
        if (!f) {
            say(" Config file %s reading failed, aborting\n", a.config.c_str());
            return kError;
        }
        text.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    }
    Config c;
    if (!read_config(text, c)) {
        say(" Config file %s reading failed, aborting\n", a.config.c_str());
        return kError;
    }
    say(" Config file %s read\n", a.config.c_str());
    // command-line overrides (src/esp.cu:497-570)
    if (a.has_gpu)
        c.v["GPU_ID_N"] = I(a.gpu);
    if (a.has_out)
        c.v["results_path"] = S(a.out.c_str());
    if (a.has_steps)
        c.v["num_steps"] = I(a.steps);
    std::string start_file;
    if (a.has_init) {
        c.v["rest"] = B(false);
        start_file  = a.initial;
    }
    if (a.has_cont) {
        if (a.batch) {
            say("--continue and --batch options set, options are exclusive, must set only one\n");
            return kError;
        }
        if (a.has_init) {
            say("--continue and --initial options set, options are exclusive, must set only one\n");
            return kError;
        }
        c.v["rest"] = B(false);
        start_file  = a.cont;
    }
    if (!c.b("rest") && start_file.empty())
        start_file = c.s("initial");
    if (!check_config(c))
        return kError;
    if (a.dump) {
        dump_config(c);
        return 0;
    }
    if (!start_file.empty() && !fs::exists(start_file)) {
        say("Initial conditions file \"%s\" not found\n", start_file.c_str());
        return kError;
    }
    const std::string out_dir = c.s("results_path"), sim_id = c.s("simulation_ID");
    std::error_code   ec;
    fs::create_directories(out_dir, ec);
    bool      continuing = a.has_cont;
    int       first_idx  = 0;
    long long step_idx   = 1;
    double    sim_time0  = 0.0;
    if (a.batch) {
        int         idx;
        long long   step;
        std::string name;
        if (last_output(out_dir, sim_id, idx, step, name)) {
            start_file = join(out_dir, name);
            continuing = true;
            say("continuing batch run from file %s\n", start_file.c_str());
        }
        else
            say("No batch file found, initialise simulation.\n");
    }
    if (!continuing && !a.overwrite && fs::exists(join(out_dir, output_name(sim_id, 0)))) {
        say("output files already exist in %s; use -w to overwrite\n", out_dir.c_str());
        return kError;
    }
    if (!start_file.empty() && start_file.size() >= 3
        && start_file.compare(start_file.size() - 3, 3, ".h5") == 0) {
        const std::string pf = planet_file(start_file, continuing);
        if (pf.empty()) {
            say("Loading initial conditions: Could not recognise file numbering scheme for input "
                "%s\n",
                start_file.c_str());
            return kError;
        }
        if (!fs::exists(pf)) {
            say("planet_file %s not found.\n", pf.c_str());
            return kError;
        }
        if (!check_planet(pf, c))
            return kError;
    }
    // the device: GPU_ID_N (or -g) through CUDA_VISIBLE_DEVICES, before the first CUDA call
    if (std::getenv("CUDA_VISIBLE_DEVICES")) {
        if (c.i("GPU_ID_N") != 0)
            say("WARNING: CUDA_VISIBLE_DEVICES is set; GPU_ID_N = %lld ignored\n", c.i("GPU_ID_N"));
    }
    else
        setenv("CUDA_VISIBLE_DEVICES", std::to_string(c.i("GPU_ID_N")).c_str(), 1);

    Grid grid;
    if (int rc = thorx_grid_build((int)c.i("glevel"), (int)c.i("vlevel"), c.d("radius"),
                                  c.d("Top_altitude"), c.b("spring_dynamics"), c.d("spring_beta"),
                                  &grid.g)) {
        say("thorx_grid_build failed (%d)\n", rc);
        return kError;
    }
    int point_num = 0, nv = 0, nl = 0, nr = 0, iters = 0;
    thorx_grid_info(grid.g, &point_num, &nv, &nl, &nr, &iters);
    thorx_grid gd{};
    thorx_grid_describe(grid.g, &gd);
    Sim                x;
    const thorx_params p = dycore_params(c);
    if (int rc = thorx_create(&gd, &p, nullptr, &x.x)) {
        say("thorx_create failed (%d): %s\n", rc, x.x ? thorx_last_error(x.x) : "");
        return kError;
    }
    struct sigaction sa {}, old_term {}, old_int {};
    bool             handlers = false;
    try {
        if (!start_file.empty()) {
            Start st;
            if (!read_state(start_file, st))
                return kError;
            std::string missing;
            for (const char* f : {"Rho", "pressure", "Mh", "Wh"})
                if (!st.fields.count(f))
                    missing += (missing.empty() ? "" : ", ") + std::string(f);
            if (!missing.empty()) {
                say("start file %s lacks %s\n", start_file.c_str(), missing.c_str());
                return kError;
            }
            const long cells = x.size("Rho");
            if (!st.fields.count("Rd")) // files without the gas constants
                st.fields["Rd"] = std::vector<double>((size_t)cells, c.d("Rd"));
            if (!st.fields.count("Cp"))
                st.fields["Cp"] = std::vector<double>((size_t)cells, c.d("Cp"));
            for (const auto& kv : st.fields)
                x.set(kv.first.c_str(), kv.second);
            sim_time0 = st.time;
            if (continuing) {
                step_idx = st.nstep + 1;
                static const std::regex re_idx("_(\\d+)\\.(h5|npz)$");
                std::smatch             m;
                first_idx = std::regex_search(start_file, m, re_idx) ? std::atoi(m[1].str().c_str()) + 1
                                                                     : 1;
            }
        }
        else if (c.s("init_PT_profile") == "guillot")
            x.check(thorx_init_guillot_state(x.x, c.d("Tmean"), c.d("Tint"), c.d("f_lw"),
                                             c.d("kappa_sw"), c.d("kappa_lw"), 0, 0.0),
                    "thorx_init_guillot_state");
        else
            x.check(thorx_init_rest_state(x.x, c.d("Tmean"), 0, 0.0), "thorx_init_rest_state");
        const bool rt = c.b("radiative_transfer");
        if (rt) {
            const thorx_rt_params r = rt_params(c, (int)step_idx);
            x.check(thorx_rt_enable(x.x, &r), "thorx_rt_enable");
        }
        if (c.b("conv_adj"))
            x.check(thorx_conv_adj_enable(x.x, (int)c.i("conv_adj_iter"), c.b("soft_adjustment")),
                    "thorx_conv_adj_enable");
        if (c.b("RayleighSponge")) {
            const thorx_sponge_params s = sponge_params(c, (int)step_idx);
            x.check(thorx_sponge_enable(x.x, &s), "thorx_sponge_enable");
        }
        if (c.b("VertHyDiff"))
            x.check(thorx_vert_hydiff_enable(x.x, c.d("Diffc_v"), (int)c.i("VertHyDiffOrder")),
                    "thorx_vert_hydiff_enable");
        const long long nsmax    = c.i("num_steps");
        const bool      globdiag = c.b("globdiag");
        Logs            logs(out_dir, sim_id, continuing, globdiag);
        write_grid(join(out_dir, "esp_output_grid_" + sim_id + ".h5"), grid, point_num, nv);
        write_planet(join(out_dir, "esp_output_planet_" + sim_id + ".h5"), c);
        const long                       ncell = x.size("Rho");
        std::vector<std::vector<double>> cells(6, std::vector<double>((size_t)ncell));
        double                           glob[6];
        auto globdiag_fields = [&]() {
            double* ptrs[6];
            for (int k = 0; k < 6; k++)
                ptrs[k] = cells[k].data();
            x.check(thorx_globdiag_fields(x.x, glob, ptrs), "thorx_globdiag_fields");
        };
        if (!continuing) {
            const std::string name = output_name(sim_id, 0);
            if (globdiag)
                globdiag_fields();
            write_state(join(out_dir, name), x, 0, sim_time0, globdiag ? glob : nullptr,
                        globdiag ? &cells : nullptr, rt);
            logs.output(0, 0, name);
            first_idx = 1;
        }
        g_caught.store(0);
        sa.sa_handler = on_signal;
        sigemptyset(&sa.sa_mask);
        sigaction(SIGTERM, &sa, &old_term);
        sigaction(SIGINT, &sa, &old_int);
        handlers               = true;
        const long long dt     = c.i("timestep");
        const long long n_out  = c.i("n_out");
        const long long g_out  = c.b("custom_global_n_out") ? c.i("global_n_out") : n_out;
        const long long l_out  = c.b("custom_log_n_out") ? c.i("log_n_out") : n_out;
        int             idx    = first_idx;
        long long       nstep  = step_idx - 1;
        const auto      t0     = std::chrono::steady_clock::now();
        say(" Starting the model integration.\n\n");
        while (nstep < nsmax) {
            // next step at which something is written: run up to it as one call (graph replays)
            long long nxt = std::min(nsmax, nstep + 64);
            for (long long k : {n_out, g_out, l_out})
                nxt = std::min(nxt, (nstep / k + 1) * k);
            const int k = (int)(nxt - nstep);
            if (c.b("gcm_off"))
                for (int s = 0; s < k; s++)
                    x.check(thorx_profx(x.x), "thorx_profx");
            else
                x.check(thorx_step(x.x, k), "thorx_step");
            x.check(thorx_sync(x.x), "thorx_sync");
            nstep                 = nxt;
            const double sim_time = sim_time0 + (double)(nstep - step_idx + 1) * (double)dt;
            const bool   writing  = nstep % n_out == 0 || g_caught.load() != 0;
            if (globdiag) {
                if (writing)
                    globdiag_fields();
                else
                    x.check(thorx_globdiag(x.x, glob), "thorx_globdiag");
                if (nstep % g_out == 0)
                    logs.globdiag(nstep, sim_time, glob);
            }
            if (writing) {
                const std::string name = output_name(sim_id, idx);
                write_state(join(out_dir, name), x, nstep, sim_time, globdiag ? glob : nullptr,
                            globdiag ? &cells : nullptr, rt);
                logs.output(nstep, idx, name);
                idx++;
            }
            const double elapsed =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            const long long done = nstep - step_idx + 1;
            const double    mean = elapsed / (double)done;
            const double    left = mean * (double)(nsmax - nstep);
            const std::time_t endt = std::time(nullptr) + (std::time_t)left;
            char              end[64];
            std::strftime(end, sizeof end, "%Y-%m-%d %H:%M:%S", std::localtime(&endt));
            if (nstep % l_out == 0) {
                say("\n Time step number = %lld/%lld || Time = %f days. \n\t Elapsed %.0f s || "
                    "Left: %.0f s || Completion: %s. \n",
                    nstep, nsmax, sim_time / 86400.0, elapsed, left, end);
                logs.diagnostics(nstep, sim_time, elapsed, left, mean, end);
            }
            if (g_caught.load()) {
                say("\n Caught signal, stopping after step %lld.\n", nstep);
                break;
            }
        }
    }
    catch (const Failure& f) {
        if (handlers) {
            sigaction(SIGTERM, &old_term, nullptr);
            sigaction(SIGINT, &old_int, nullptr);
        }
        say("%s\n", f.what.c_str());
        return kError;
    }
    if (handlers) {
        sigaction(SIGTERM, &old_term, nullptr);
        sigaction(SIGINT, &old_int, nullptr);
    }
    return 0;
}

} // namespace

int main(int argc, char** argv) { return run(argc, argv); }
