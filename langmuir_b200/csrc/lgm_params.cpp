// lgm_params.cpp -- Langmuir input keys: defaults, parser, validation.
//
// Same keys, defaults and checks as the reference (keyvalueparser.cpp:15-173,
// include/parameters.h:285-646, include/variable.h:267-276, 330-350), with
// status codes and messages where the reference called qFatal.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "langmuir_b200_kmc.h"

namespace {

enum Kind { K_STR16, K_STR64, K_U32, K_U64, K_I32, K_BOOL, K_F64 };
struct Key {
    const char* name;
    Kind kind;
    size_t offset;
    bool constant;
};

#define K(name, kind, field) {name, kind, offsetof(lgm_params, field), false}
#define KC(name, kind, field) {name, kind, offsetof(lgm_params, field), true}

// Registration order of KeyValueParser::KeyValueParser (keyvalueparser.cpp:15-105),
// then the two extension keys.
const Key kKeys[] = {
    K("simulation.type", K_STR16, simulation_type),
    K("current.step", K_U32, current_step),
    K("iterations.real", K_I32, iterations_real),
    K("random.seed", K_U64, random_seed),
    K("grid.z", K_I32, grid_z), K("grid.y", K_I32, grid_y), K("grid.x", K_I32, grid_x),
    K("hopping.range", K_I32, hopping_range),
    K("output.is.on", K_BOOL, output_is_on),
    K("iterations.print", K_I32, iterations_print),
    K("output.precision", K_I32, output_precision),
    K("output.width", K_I32, output_width),
    K("output.stub", K_STR64, output_stub),
    K("output.ids.on.delete", K_BOOL, output_ids_on_delete),
    K("output.ids.on.encounter", K_BOOL, output_ids_on_encounter),
    K("output.coulomb", K_I32, output_coulomb),
    K("output.step.chk", K_I32, output_step_chk),
    K("output.chk.trap.potential", K_BOOL, output_chk_trap_potential),
    K("output.potential", K_BOOL, output_potential),
    K("output.xyz", K_I32, output_xyz),
    K("output.xyz.e", K_BOOL, output_xyz_e), K("output.xyz.h", K_BOOL, output_xyz_h),
    K("output.xyz.d", K_BOOL, output_xyz_d), K("output.xyz.t", K_BOOL, output_xyz_t),
    K("output.xyz.mode", K_I32, output_xyz_mode),
    K("image.traps", K_BOOL, image_traps), K("image.defects", K_BOOL, image_defects),
    K("image.carriers", K_I32, image_carriers),
    K("electron.percentage", K_F64, electron_percentage),
    K("hole.percentage", K_F64, hole_percentage),
    K("seed.charges", K_F64, seed_charges),
    K("defect.percentage", K_F64, defect_percentage),
    K("trap.percentage", K_F64, trap_percentage),
    K("trap.potential", K_F64, trap_potential),
    K("gaussian.stdev", K_F64, gaussian_stdev),
    K("seed.percentage", K_F64, seed_percentage),
    K("voltage.right", K_F64, voltage_right), K("voltage.left", K_F64, voltage_left),
    K("slope.z", K_F64, slope_z),
    K("coulomb.carriers", K_BOOL, coulomb_carriers),
    K("coulomb.gaussian.sigma", K_F64, coulomb_gaussian_sigma),
    K("defects.charge", K_I32, defects_charge),
    K("exciton.binding", K_F64, exciton_binding),
    K("temperature.kelvin", K_F64, temperature_kelvin),
    K("source.rate", K_F64, source_rate),
    K("e.source.l.rate", K_F64, e_source_l_rate), K("e.source.r.rate", K_F64, e_source_r_rate),
    K("h.source.l.rate", K_F64, h_source_l_rate), K("h.source.r.rate", K_F64, h_source_r_rate),
    K("generation.rate", K_F64, generation_rate),
    K("source.metropolis", K_BOOL, source_metropolis),
    K("source.coulomb", K_BOOL, source_coulomb),
    K("source.scale.area", K_F64, source_scale_area),
    K("balance.charges", K_BOOL, balance_charges),
    K("drain.rate", K_F64, drain_rate),
    K("e.drain.l.rate", K_F64, e_drain_l_rate), K("e.drain.r.rate", K_F64, e_drain_r_rate),
    K("h.drain.l.rate", K_F64, h_drain_l_rate), K("h.drain.r.rate", K_F64, h_drain_r_rate),
    K("recombination.rate", K_F64, recombination_rate),
    K("recombination.range", K_I32, recombination_range),
    K("use.opencl", K_BOOL, use_opencl),
    K("work.x", K_I32, work_x), K("work.y", K_I32, work_y), K("work.z", K_I32, work_z),
    K("work.size", K_I32, work_size),
    K("opencl.threshold", K_I32, opencl_threshold),
    K("opencl.device.id", K_I32, opencl_device_id),
    K("max.threads", K_I32, max_threads),
    KC("boltzmann.constant", K_F64, boltzmann_constant),
    KC("dielectric.constant", K_F64, dielectric_constant),
    KC("elementary.charge", K_F64, elementary_charge),
    KC("permittivity.space", K_F64, permittivity_space),
    KC("grid.factor", K_F64, grid_factor),
    KC("electrostatic.cutoff", K_I32, electrostatic_cutoff),
    KC("electrostatic.prefactor", K_F64, electrostatic_prefactor),
    KC("inverse.kt", K_F64, inverse_kt),
    KC("ok.cl", K_BOOL, use_opencl),           // constant: never written
    KC("simulation.start", K_STR64, output_stub),  // constant: never written
    K("image.charges", K_I32, image_charges),
    K("site.disorder", K_F64, site_disorder),
    K("morphology.confine", K_BOOL, morphology_confine),
    K("generation.interface", K_BOOL, generation_interface),
};

void set_err(char* err, int len, const std::string& m) {
    if (err && len > 0) {
        std::snprintf(err, (size_t)len, "%s", m.c_str());
    }
}

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// TypedVariable<T>::convert (variable.h:310-400): numbers must parse whole;
// bools accept true/false (any case) or an integer.
bool convert(const Key& k, const std::string& tok, lgm_params* p, std::string* why) {
    unsigned char* base = reinterpret_cast<unsigned char*>(p) + k.offset;
    const char* s = tok.c_str();
    char* end = nullptr;
    errno = 0;
    switch (k.kind) {
    case K_STR16:
    case K_STR64: {
        const size_t cap = k.kind == K_STR16 ? 16 : 64;
        if (tok.size() >= cap) { *why = "string too long"; return false; }
        std::memset(base, 0, cap);
        std::memcpy(base, tok.data(), tok.size());
        return true;
    }
    case K_U32:
    case K_U64: {
        if (!tok.empty() && tok[0] == '-') { *why = "can not convert to unsigned int"; return false; }
        unsigned long long v = std::strtoull(s, &end, 10);
        if (end == s || *end || errno) { *why = "can not convert to unsigned int"; return false; }
        if (k.kind == K_U32) {
            if (v > 0xffffffffull) { *why = "out of range"; return false; }
            *reinterpret_cast<uint32_t*>(base) = (uint32_t)v;
        } else {
            *reinterpret_cast<uint64_t*>(base) = v;
        }
        return true;
    }
    case K_I32: {
        long v = std::strtol(s, &end, 10);
        if (end == s || *end || errno || v < INT32_MIN || v > INT32_MAX) {
            *why = "can not convert to int";
            return false;
        }
        *reinterpret_cast<int32_t*>(base) = (int32_t)v;
        return true;
    }
    case K_BOOL: {
        const std::string l = lower(tok);
        if (l == "false") { *reinterpret_cast<int32_t*>(base) = 0; return true; }
        if (l == "true") { *reinterpret_cast<int32_t*>(base) = 1; return true; }
        long v = std::strtol(s, &end, 10);
        if (end == s || *end) { *why = "can not convert to bool"; return false; }
        *reinterpret_cast<int32_t*>(base) = v != 0;
        return true;
    }
    case K_F64: {
        double v = std::strtod(s, &end);
        if (end == s || *end) { *why = "can not convert to double"; return false; }
        *reinterpret_cast<double*>(base) = v;
        return true;
    }
    }
    return false;
}

}  // namespace

extern "C" {

int32_t lgm_params_size(void) { return (int32_t)sizeof(lgm_params); }

void lgm_params_default(lgm_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    // SimulationParameters() (parameters.h:285-378)
    std::snprintf(p->simulation_type, sizeof p->simulation_type, "transistor");
    p->random_seed = 0;
    p->grid_z = 1; p->grid_y = 128; p->grid_x = 128;
    p->coulomb_carriers = 0; p->coulomb_gaussian_sigma = 0.0; p->defects_charge = 0;
    p->output_xyz = 0; p->output_xyz_e = p->output_xyz_h = p->output_xyz_d = p->output_xyz_t = 1;
    p->output_xyz_mode = 0;
    p->output_ids_on_delete = 0; p->output_coulomb = 0; p->output_step_chk = 1;
    p->output_chk_trap_potential = 0; p->output_potential = 0; p->output_is_on = 1;
    p->image_defects = 0; p->image_traps = 0; p->image_carriers = 0;
    p->iterations_print = 10; p->iterations_real = 1000;
    p->output_precision = 15; p->output_width = 23;
    std::snprintf(p->output_stub, sizeof p->output_stub, "out");
    p->electron_percentage = 0.01; p->hole_percentage = 0.0; p->seed_charges = 0.0;
    p->defect_percentage = 0.0; p->trap_percentage = 0.0; p->trap_potential = 0.10;
    p->gaussian_stdev = 0.0; p->seed_percentage = 1.0;
    p->voltage_right = 0.0; p->voltage_left = 0.0; p->exciton_binding = 0.0;
    p->temperature_kelvin = 300.0;
    p->source_rate = 0.90;
    p->e_source_l_rate = p->e_source_r_rate = p->h_source_l_rate = p->h_source_r_rate = -1.0;
    p->generation_rate = 0.001; p->balance_charges = 0;
    p->drain_rate = 0.90;
    p->e_drain_l_rate = p->e_drain_r_rate = p->h_drain_l_rate = p->h_drain_r_rate = -1.0;
    p->use_opencl = 0; p->work_x = p->work_y = p->work_z = 4; p->work_size = 256;
    p->opencl_threshold = 256; p->opencl_device_id = 0;
    p->boltzmann_constant = 1.3806504e-23; p->dielectric_constant = 3.5;
    p->elementary_charge = 1.60217646e-19; p->permittivity_space = 8.854187817e-12;
    p->grid_factor = 1e-9; p->electrostatic_cutoff = 50;
    p->electrostatic_prefactor = 0; p->inverse_kt = 0;
    p->current_step = 0; p->hopping_range = 1; p->slope_z = 0.0;
    p->source_metropolis = 0; p->source_coulomb = 0;
    p->recombination_rate = 0.0; p->recombination_range = 0;
    p->output_ids_on_encounter = 0; p->source_scale_area = 65536; p->max_threads = -1;
    p->image_charges = 0; p->site_disorder = 0.0;
    p->guard_band = LGM_GUARD_BAND_MIN;
}

lgm_status lgm_params_parse(const char* text, lgm_params* p, char* err, int32_t err_len) {
    if (!text || !p) return LGM_ERR_INVALID_ARGUMENT;
    std::string all(text);
    size_t pos = 0;
    // CheckPointer::load reads a section header first (checkpointer.cpp:44-70).
    {
        size_t a = all.find_first_not_of(" \t\r\n");
        if (a == std::string::npos) return LGM_OK;
        size_t b = all.find_first_of(" \t\r\n", a);
        std::string head = all.substr(a, b == std::string::npos ? std::string::npos : b - a);
        std::string sec;
        for (char c : head)
            if (c != '[' && c != ']') sec += c;
        if (sec != "Parameters") {
            set_err(err, err_len, "langmuir: invalid section encountered: " + sec +
                                      " (the first section must be [Parameters])");
            return LGM_ERR_PARSE;
        }
        // the rest of the header line is consumed by the next getline
        pos = b == std::string::npos ? all.size() : b;
    }
    // loadParameters: getline until "end"; a final line without '\n' is not
    // parsed (std::getline sets eof on it, checkpointer.cpp:408-414).
    while (pos < all.size()) {
        size_t nl = all.find('\n', pos);
        if (nl == std::string::npos) break;
        std::string raw = all.substr(pos, nl - pos);
        pos = nl + 1;
        std::string line = trim(raw);
        if (lower(line) == "end") break;
        // KeyValueParser::parse (keyvalueparser.cpp:112-173)
        size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        line = trim(line);
        if (line.empty()) continue;
        if (std::count(line.begin(), line.end(), '=') != 1) {
            set_err(err, err_len, "langmuir: parse error: missing equal sign\n\tline: " + trim(raw));
            return LGM_ERR_PARSE;
        }
        const size_t eq = line.find('=');
        const std::string key = lower(trim(line.substr(0, eq)));
        std::string value = trim(line.substr(eq + 1));
        if (key.empty()) {
            set_err(err, err_len, "langmuir: parse error: key is empty\n\tline: " + trim(raw));
            return LGM_ERR_PARSE;
        }
        const Key* k = nullptr;
        for (const Key& c : kKeys)
            if (key == c.name) { k = &c; break; }
        if (!k) {
            set_err(err, err_len, "langmuir: parse error: invalid key\n\tline: " + trim(raw));
            return LGM_ERR_PARSE;
        }
        while (!value.empty() && value.front() == '"') value.erase(value.begin());
        while (!value.empty() && value.back() == '"') value.pop_back();
        if (value.empty()) continue;  // "warning! value is empty" -- not an error
        if (k->constant) continue;    // variable.h:269-274: constants are ignored
        std::string why;
        if (!convert(*k, value, p, &why)) {
            set_err(err, err_len, "langmuir: " + why + ": " + value + " (key " + key + ")");
            return LGM_ERR_PARSE;
        }
    }
    return LGM_OK;
}

lgm_status lgm_params_check(lgm_params* p, char* err, int32_t err_len) {
    if (!p) return LGM_ERR_INVALID_ARGUMENT;
    // setCalculatedValues (parameters.h:384-390)
    p->electrostatic_prefactor = p->elementary_charge /
                                 (4.0 * M_PI * p->dielectric_constant * p->permittivity_space *
                                  p->grid_factor);
    p->inverse_kt = p->elementary_charge / (p->boltzmann_constant * p->temperature_kelvin);
    if (p->output_width < 8) p->output_width = 8;
    if (p->output_width < p->output_precision + 8) p->output_width = p->output_precision + 8;
    char b[256];
    auto bad = [&](const char* fmt, double a = 0, double c = 0) {
        std::snprintf(b, sizeof b, fmt, a, c);
        set_err(err, err_len, std::string("langmuir: ") + b);
        return LGM_ERR_INVALID_ARGUMENT;
    };
    const std::string st = p->simulation_type;
    if (st != "transistor" && st != "solarcell")
        return bad("simulation.type must be transistor or solarcell");
    if (p->grid_z < 1 || p->grid_y < 1 || p->grid_x < 1) return bad("grid.x, grid.y, grid.z >= 1");
    if (p->iterations_print <= 0) return bad("iterations.print(%g) <= 0", p->iterations_print);
    if (p->iterations_real < 0) return bad("iterations.real(%g) < 0", p->iterations_real);
    if (p->iterations_real % p->iterations_print != 0)
        return bad("iterations.real(%g) %% iterations.print(%g) != 0", p->iterations_real,
                   p->iterations_print);
    auto frac = [](double v) { return v < 0.0 || v > 1.0; };
    if (frac(p->electron_percentage)) return bad("electron.pecentage(%f) < 0 || > 1.0", p->electron_percentage);
    if (frac(p->hole_percentage)) return bad("hole.pecentage(%f) < 0 || > 1.0", p->hole_percentage);
    if (frac(p->defect_percentage)) return bad("defect.pecentage(%f) < 0 || > 1.0", p->defect_percentage);
    if (frac(p->trap_percentage)) return bad("trap.pecentage(%f) < 0 || > 1.0", p->trap_percentage);
    if (frac(p->seed_percentage)) return bad("seed.pecentage(%f) < 0 || > 1.0", p->seed_percentage);
    if (p->defect_percentage > 1.00 - p->trap_percentage)
        return bad("trap.percentage(%f) > 1.0 - trap.percentage(%f)", p->defect_percentage,
                   p->trap_percentage);
    if (frac(p->source_rate)) return bad("source.rate(%f) < 0 || > 1.0", p->source_rate);
    const double rates[] = {p->e_source_l_rate, p->e_source_r_rate, p->h_source_l_rate,
                            p->h_source_r_rate, p->generation_rate, p->e_drain_l_rate,
                            p->e_drain_r_rate, p->h_drain_l_rate, p->h_drain_r_rate};
    for (double r : rates)
        if (r >= 0.0 && r > 1.0) return bad("a source or drain rate (%f) is > 1.0", r);
    if (frac(p->drain_rate)) return bad("drain.rate(%f) < 0 || > 1.0", p->drain_rate);
    if (frac(p->seed_charges)) return bad("seed.charges(%f) < 0 || > 1.0", p->seed_charges);
    if (p->gaussian_stdev < 0.0) return bad("gaussian.stdev < 0.0");
    if (p->temperature_kelvin < 0.0) return bad("temperature.kelvin < 0.0");
    if (p->defects_charge != 0 && !p->coulomb_carriers)
        return bad("defects.charge != 0 && coulomb.carriers = false");
    if (p->hopping_range < 0 || p->hopping_range > 2)
        return bad("hopping.range(%g) < 0 || > 2", p->hopping_range);
    if (!p->source_metropolis && p->source_coulomb)
        return bad("source.metropolis = false, yet source.coulomb = true");
    if (frac(p->recombination_rate)) return bad("recombination.rate(%f) < 0 || > 1.0", p->recombination_rate);
    if (p->recombination_rate > 0 && st != "solarcell")
        return bad("recombination.rate(%f) > 0, yet simulation.type != solarcell", p->recombination_rate);
    if (p->recombination_rate > 0 && !(p->electron_percentage > 0 && p->hole_percentage > 0))
        return bad("recombination.rate > 0, yet electron.percentage or hole.percentage is 0");
    if (p->output_ids_on_encounter && st != "solarcell")
        return bad("output.ids.on.encounter == true, yet simulation.type != solarcell");
    if (!p->output_xyz_e && !p->output_xyz_h && !p->output_xyz_d && !p->output_xyz_t &&
        p->output_xyz > 0)
        return bad("output.xyz > 0, yet output.xyz.e/h/d/t are all false");
    if (p->output_xyz_mode < 0 || p->output_xyz_mode > 1) return bad("output.xyz.mode must be 0 or 1");
    if (p->opencl_threshold <= 0) return bad("opencl.threshold must be >= 0");
    if (p->opencl_device_id < 0) return bad("opencl.device.id must be >= 0");
    if (p->balance_charges && st != "solarcell")
        return bad("balance.charges == true, yet simulation.type != solarcell");
    if (p->coulomb_gaussian_sigma > 0 && (p->grid_x == 1 || p->grid_y == 1 || p->grid_z == 1))
        return bad("coulomb.gaussian.sigma > 0, yet the simulation is not 3D");
    if (p->output_ids_on_encounter) return bad("output.ids.on.encouter is deprecated");
    if (p->image_charges < 0 || p->image_charges > 3) return bad("image.charges must be 0..3");
    if (p->site_disorder < 0) return bad("site.disorder < 0");
    if (!(p->guard_band >= LGM_GUARD_BAND_MIN) || !std::isfinite(p->guard_band))
        return bad("guard band %g below the FP32C error bound %g", p->guard_band,
                   LGM_GUARD_BAND_MIN);
    if (p->generation_interface && st != "solarcell")
        return bad("generation.interface == true, yet simulation.type != solarcell");
    return LGM_OK;
}

int32_t lgm_params_format(const lgm_params* p, char* out, int32_t cap) {
    if (!p) return -1;
    std::string text = "[Parameters]";
    const size_t n_reference = sizeof(kKeys) / sizeof(kKeys[0]) - 4;  // the extension keys last
    for (size_t i = 0; i < sizeof(kKeys) / sizeof(kKeys[0]); ++i) {
        const Key& k = kKeys[i];
        if (k.constant) continue;
        const char* base = reinterpret_cast<const char*>(p) + k.offset;
        std::string value;
        char buf[64];
        switch (k.kind) {
        case K_STR16:
            value.assign(base, strnlen(base, 16));
            break;
        case K_STR64:
            value.assign(base, strnlen(base, 64));
            break;
        case K_U32:
            std::snprintf(buf, sizeof buf, "%u", *reinterpret_cast<const uint32_t*>(base));
            value = buf;
            break;
        case K_U64:
            std::snprintf(buf, sizeof buf, "%llu",
                          (unsigned long long)*reinterpret_cast<const uint64_t*>(base));
            value = buf;
            break;
        case K_I32:
            std::snprintf(buf, sizeof buf, "%d", *reinterpret_cast<const int32_t*>(base));
            value = buf;
            break;
        case K_BOOL:
            value = *reinterpret_cast<const int32_t*>(base) ? "True" : "False";
            break;
        case K_F64:
            // TypedVariable<qreal>::value: scientific, digits10 = 15 digits
            std::snprintf(buf, sizeof buf, "%.15e", *reinterpret_cast<const double*>(base));
            value = buf;
            break;
        }
        // extension keys only when set, so that the reference can read the text
        if (i >= n_reference && (value == "0" || value == "False" ||
                                 (k.kind == K_F64 && *reinterpret_cast<const double*>(base) == 0.0)))
            continue;
        // TypedVariable::keyValue (variable.h:196-238): key left in 30 columns,
        // '=' in 3 columns (2 before a minus sign), then the value
        std::string line = k.name;
        if (line.size() < 30) line.append(30 - line.size(), ' ');
        if (value.empty()) line += "=";
        else line += (value[0] == '-' ? "= " : "=  ") + value;
        text += "\n" + line;
    }
    text += "\n";
    const int32_t need = (int32_t)text.size() + 1;
    if (out && cap > 0) std::snprintf(out, (size_t)cap, "%s", text.c_str());
    return need;
}

}  // extern "C"
