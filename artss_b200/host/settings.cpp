#include "settings.h"

#include <algorithm>
#include <cctype>
#include <fstream>
#include <map>
#include <sstream>

#include "xml.h"

namespace artss {

const char *const kPatchNames[kPatches] = {"left", "right", "bottom", "top", "front", "back"};
const char *const kFieldTypeNames[kFieldTypesHost] = {"rho", "u", "v", "w", "p", "T", "nu"};

namespace settings {
namespace {

using Map = std::map<std::string, std::string>;
const char *const kYes = "Yes";

// Section `name` among the children of `head`: its attributes plus the text
// of its children (Settings.cpp:23-55, map_parameter_section).
struct Section {
    const XmlElement *el = nullptr;
    Map values;
};

Section section(const XmlElement *head, const std::string &name) {
    Section s;
    if (!head) return s;
    const XmlElement *e = head->first_child(name);
    if (!e) return s;
    s.el = e;
    for (const auto &kv : e->attributes) s.values[kv.first] = kv.second;
    for (const auto &c : e->children)
        if (c->has_text) s.values[c->name] = c->text;
    return s;
}

Map attributes(const XmlElement *e) {
    Map m;
    for (const auto &kv : e->attributes) m[kv.first] = kv.second;
    return m;
}

std::string ctx_join(const std::string &a, const std::string &b) { return a + "/" + b; }

[[noreturn]] void missing(const std::string &key, const std::string &context) {
    throw config_error("Value " + key + " is for " + context + " required.");
}

size_t req_size(const Map &m, const std::string &key, const std::string &context) {
    auto it = m.find(key);
    if (it == m.end()) missing(key, context);
    try {
        return static_cast<size_t>(std::stoi(it->second));
    } catch (const std::exception &) {
        missing(key, context);
    }
}

size_t opt_size(const Map &m, const std::string &key, size_t dflt) {
    auto it = m.find(key);
    return it == m.end() ? dflt : static_cast<size_t>(std::stoi(it->second));
}

double req_real(const Map &m, const std::string &key, const std::string &context) {
    auto it = m.find(key);
    if (it == m.end()) missing(key, context);
    try {
        return std::stod(it->second);
    } catch (const std::exception &) {
        missing(key, context);
    }
}

double opt_real(const Map &m, const std::string &key, double dflt) {
    auto it = m.find(key);
    return it == m.end() ? dflt : std::stod(it->second);
}

std::string req_str(const Map &m, const std::string &key, const std::string &context) {
    auto it = m.find(key);
    if (it == m.end()) missing(key, context);
    return it->second;
}

std::string opt_str(const Map &m, const std::string &key, const std::string &dflt) {
    auto it = m.find(key);
    return it == m.end() ? dflt : it->second;
}

bool req_bool(const Map &m, const std::string &key, const std::string &context) {
    return req_str(m, key, context) == kYes;
}

bool opt_bool(const Map &m, const std::string &key, bool dflt) {
    auto it = m.find(key);
    return it == m.end() ? dflt : it->second == kYes;
}

std::vector<std::string> split(const std::string &text) {
    std::vector<std::string> out;
    std::stringstream ss(text);
    std::string tok;
    while (std::getline(ss, tok, ',')) out.push_back(tok);
    return out;
}

int match_name(const std::string &s, const char *const *names, int n, const char *what) {
    for (int k = 0; k < n; k++)
        if (s == names[k]) return k;
    throw config_error(std::string("unknown ") + what + " '" + s + "'");
}

int match_field(const std::string &s) { return match_name(s, kFieldTypeNames, kFieldTypesHost, "field"); }
int match_patch(const std::string &s) { return match_name(s, kPatchNames, kPatches, "patch"); }

int match_bc(const std::string &s) {
    static const char *const names[3] = {"neumann", "dirichlet", "periodic"};
    return match_name(s, names, 3, "boundary condition");
}

// Mapping::match_axis (src/utility/Mapping.cpp:17-23): an unknown name maps to
// UNKNOWN_AXIS (-1), which the solvers then ignore
int match_axis(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char) std::toupper(c); });
    static const char *const names[3] = {"X", "Y", "Z"};
    for (int k = 0; k < 3; k++)
        if (s == names[k]) return k;
    return -1;
}

std::vector<int> fields_of(const std::string &list) {
    std::vector<int> v;
    for (auto &s : split(list)) v.push_back(match_field(s));
    return v;
}

std::vector<int> axes_of(const std::string &list) {
    std::vector<int> v;
    for (auto &s : split(list)) v.push_back(match_axis(s));
    return v;
}

const XmlElement *need(const Section &s, const std::string &context) {
    if (!s.el) throw config_error("Section " + context + " is required.");
    return s.el;
}

Random parse_random(const XmlElement *head, const std::string &parent) {
    const std::string context = ctx_join(parent, "random");
    Section s = section(head, "random");
    Random r;
    r.absolute = req_bool(s.values, "absolute", context);
    r.custom_seed = req_bool(s.values, "custom_seed", context);
    r.seed = r.custom_seed ? req_size(s.values, "seed", context) : opt_size(s.values, "seed", 0);
    r.custom_steps = req_bool(s.values, "custom_steps", context);
    r.step_size = r.custom_steps ? req_real(s.values, "step_size", context) : opt_real(s.values, "step_size", 1);
    r.range = req_real(s.values, "range", context);
    return r;
}

Boundary parse_boundary(const XmlElement *e, const std::string &parent) {
    const std::string context = ctx_join(parent, "boundary");
    Map v = attributes(e);
    Boundary b;
    b.bc = match_bc(req_str(v, "type", context));
    if (b.bc != BC_PERIODIC) b.value = req_real(v, "value", context);
    b.field_types = fields_of(req_str(v, "field", context));
    for (auto &p : split(req_str(v, "patch", context))) b.patches.push_back(match_patch(p));
    return b;
}

Advection parse_advection(const XmlElement *head, const std::string &parent) {
    const std::string context = ctx_join(parent, "advection");
    Section s = section(head, "advection");
    Advection a;
    a.type = req_str(s.values, "type", context);
    if (a.type != "SemiLagrangian")
        throw config_error("advection solver '" + a.type + "' has no parsing implementation.");
    a.fields = fields_of(req_str(s.values, "field", context));
    return a;
}

Diffusion parse_diffusion(const XmlElement *head, const std::string &parent) {
    const std::string context = ctx_join(parent, "diffusion");
    Section s = section(head, "diffusion");
    Diffusion d;
    d.type = req_str(s.values, "type", context);
    if (d.type == "Jacobi" || d.type == "ColoredGaussSeidel" || d.type == "ColoredGaussSeidelMixed") {
        const std::string c2 = ctx_join(context, d.type);
        d.has_iteration = true;
        d.w = req_real(s.values, "w", c2);
        d.tol_res = req_real(s.values, "tol_res", c2);
        d.max_iter = req_size(s.values, "max_iter", c2);
    } else if (d.type != "Explicit") {
        throw config_error("diffusion solver '" + d.type + "' has no parsing implementation.");
    }
    d.fields = fields_of(req_str(s.values, "field", context));
    return d;
}

Turbulence parse_turbulence(const XmlElement *head, const std::string &parent) {
    const std::string context = ctx_join(parent, "turbulence");
    Section s = section(head, "turbulence");
    Turbulence t;
    t.type = req_str(s.values, "type", context);
    if (t.type == "ConstSmagorinsky") {
        t.has_cs = true;
        t.cs = req_real(s.values, "Cs", ctx_join(context, "ConstSmagorinsky"));
    } else if (t.type != "DynamicSmagorinsky") {
        throw config_error("turbulence solver '" + t.type + "' has no parsing implementation.");
    }
    return t;
}

Source parse_source(const XmlElement *head, const std::string &parent) {
    const std::string context = ctx_join(parent, "source");
    Section s = section(head, "source");
    Source src;
    src.type = req_str(s.values, "type", context);
    src.force_fct = req_str(s.values, "force_fct", context);
    if (src.force_fct == "Buoyancy") {
        const std::string c2 = ctx_join(context, "Buoyancy");
        src.use_init_values = req_bool(s.values, "use_init_values", c2);
        if (!src.use_init_values) src.ambient_temperature = req_real(s.values, "ambient_temperature_value", c2);
    } else if (src.force_fct == "Uniform") {
        const std::string c2 = ctx_join(context, "Uniform");
        src.uniform_value = {req_real(s.values, "val_x", c2), req_real(s.values, "val_y", c2),
                             req_real(s.values, "val_z", c2)};
    } else if (src.force_fct != "Zero") {
        throw config_error("source type '" + src.type + "' has no parsing implementation.");
    }
    src.dir = axes_of(req_str(s.values, "dir", context));
    return src;
}

Pressure parse_pressure(const XmlElement *head, const std::string &parent) {
    const std::string context = ctx_join(parent, "pressure");
    Section s = section(head, "pressure");
    Pressure p;
    p.type = req_str(s.values, "type", context);
    p.field = match_field(req_str(s.values, "field", context));
    // VCycleMGMixed (no reference counterpart) reads the same keys; tol_res is
    // its relative tolerance and max_cycle its cycle limit per solve
    if (p.type != "VCycleMG" && p.type != "VCycleMGMixed" && p.type != "VCycleMGRel")
        throw config_error("pressure solver '" + p.type + "' has no parsing implementation.");
    const std::string c2 = ctx_join(context, "vcycle");
    p.n_level = req_size(s.values, "n_level", c2);
    p.n_cycle = req_size(s.values, "n_cycle", c2);
    p.max_cycle = req_size(s.values, "max_cycle", c2);
    p.n_relax = req_size(s.values, "n_relax", c2);
    p.tol_res = req_real(s.values, "tol_res", c2);
    p.smoother = parse_diffusion(need(s, context), c2);
    return p;
}

Gauss parse_gauss(const Map &v, const std::string &parent) {
    const std::string context = ctx_join(parent, "Gauss");
    Gauss g;
    g.heat_release_rate = req_real(v, "HRR", context);
    g.heat_capacity = req_real(v, "cp", context);
    const char *ax[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; a++) {
        g.position[a] = req_real(v, std::string(ax[a]) + "0", context);
        g.dimension[a] = req_real(v, std::string("sigma_") + ax[a], context);
    }
    g.tau = req_real(v, "tau", context);
    return g;
}

Cube parse_cube(const Map &v, const std::string &parent) {
    const std::string context = ctx_join(parent, "Cube");
    Cube c;
    const char *ax[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; a++) {
        c.start[a] = req_real(v, std::string(ax[a]) + "_start", context);
        c.end[a] = req_real(v, std::string(ax[a]) + "_end", context);
    }
    c.value = req_real(v, "val", context);
    return c;
}

TemperatureSource parse_temperature_source(const XmlElement *head, const std::string &parent) {
    const std::string context = ctx_join(parent, "source");
    Section s = section(head, "source");
    TemperatureSource t;
    t.type = req_str(s.values, "type", context);
    t.dir = axes_of(req_str(s.values, "dir", context));
    t.dissipation = req_bool(s.values, "dissipation", context);
    t.random = req_bool(s.values, "random", context);
    if (t.random) t.random_parameters = parse_random(need(s, context), context);
    t.temp_fct = req_str(s.values, "temp_fct", context);
    if (t.temp_fct == "Gauss") t.gauss = parse_gauss(s.values, context);
    else if (t.temp_fct == "Cube") t.cube = parse_cube(s.values, context);
    else if (t.temp_fct != "Buoyancy" && t.temp_fct != "Zero")
        throw config_error("temperature source function '" + t.temp_fct + "' has no parsing implementation.");
    return t;
}

Temperature parse_temperature(const XmlElement *head, const std::string &parent, bool turbulence) {
    const std::string context = ctx_join(parent, "temperature");
    Section s = section(head, "temperature");
    const XmlElement *sub = need(s, context);
    Temperature t;
    t.advection = parse_advection(sub, context);
    t.diffusion = parse_diffusion(sub, context);
    if (turbulence) {
        Section ts = section(sub, "turbulence");
        const std::string c2 = ctx_join(context, "turbulence");
        t.has_turbulence = req_bool(ts.values, "include", c2);
        if (t.has_turbulence) t.prandtl_number = req_real(ts.values, "Pr_T", c2);
    }
    t.source = parse_temperature_source(sub, context);
    return t;
}

// Settings.cpp:840-889
Concentration parse_concentration(const XmlElement *head, const std::string &parent, bool turbulence) {
    const std::string context = ctx_join(parent, "concentration");
    Section s = section(head, "concentration");
    const XmlElement *sub = need(s, context);
    Concentration c;
    c.advection = parse_advection(sub, context);
    c.diffusion = parse_diffusion(sub, context);
    if (turbulence) {
        Section ts = section(sub, "turbulence");
        const std::string c2 = ctx_join(context, "turbulence");
        c.has_turbulence = req_bool(ts.values, "include", c2);
        if (c.has_turbulence) c.turbulent_schmidt_number = req_real(ts.values, "Sc_T", c2);
    }
    Section ss = section(sub, "source");
    const std::string cs = "source";
    c.source.type = req_str(ss.values, "type", cs);
    c.source.dir = axes_of(req_str(ss.values, "dir", cs));
    c.source.random = req_bool(ss.values, "random", cs);
    if (c.source.random) c.source.random_parameters = parse_random(need(ss, ctx_join(context, cs)), ctx_join(context, cs));
    c.source.con_fct = req_str(ss.values, "con_fct", cs);
    if (c.source.con_fct == "Gauss") c.source.gauss = parse_gauss(ss.values, cs);
    else if (c.source.con_fct == "Cube") c.source.cube = parse_cube(ss.values, cs);
    else
        throw config_error("concentration source function '" + c.source.con_fct + "' has no parsing implementation.");
    return c;
}

Solver parse_solver(const XmlElement *root) {
    const std::string context = "solver";
    Section s = section(root, context);
    Solver sp;
    sp.description = req_str(s.values, "description", context);
    const XmlElement *sub = need(s, context);
    const std::string &d = sp.description;
    if (d == "AdvectionSolver") {
        sp.advection = parse_advection(sub, context);
    } else if (d == "AdvectionDiffusionSolver") {
        sp.advection = parse_advection(sub, context);
        sp.diffusion = parse_diffusion(sub, context);
    } else if (d == "DiffusionSolver") {
        sp.diffusion = parse_diffusion(sub, context);
    } else if (d == "DiffusionTurbSolver") {
        sp.diffusion = parse_diffusion(sub, context);
        sp.turbulence = parse_turbulence(sub, context);
    } else if (d == "NSSolver") {
        sp.advection = parse_advection(sub, context);
        sp.diffusion = parse_diffusion(sub, context);
        sp.pressure = parse_pressure(sub, context);
        sp.source = parse_source(sub, context);
    } else if (d == "NSTempSolver") {
        sp.advection = parse_advection(sub, context);
        sp.diffusion = parse_diffusion(sub, context);
        sp.pressure = parse_pressure(sub, context);
        sp.temperature = parse_temperature(sub, context, false);
        sp.source = parse_source(sub, context);
    } else if (d == "NSTempTurbSolver") {
        sp.advection = parse_advection(sub, context);
        sp.diffusion = parse_diffusion(sub, context);
        sp.pressure = parse_pressure(sub, context);
        sp.temperature = parse_temperature(sub, context, true);
        sp.turbulence = parse_turbulence(sub, context);
        sp.source = parse_source(sub, context);
    } else if (d == "NSTempConSolver") {
        sp.advection = parse_advection(sub, context);
        sp.diffusion = parse_diffusion(sub, context);
        sp.pressure = parse_pressure(sub, context);
        sp.temperature = parse_temperature(sub, context, false);
        sp.concentration = parse_concentration(sub, context, false);
        sp.source = parse_source(sub, context);
    } else if (d == "NSTempTurbConSolver") {
        sp.advection = parse_advection(sub, context);
        sp.diffusion = parse_diffusion(sub, context);
        sp.pressure = parse_pressure(sub, context);
        sp.temperature = parse_temperature(sub, context, true);
        sp.turbulence = parse_turbulence(sub, context);
        sp.concentration = parse_concentration(sub, context, true);
        sp.source = parse_source(sub, context);
    } else if (d == "NSTurbSolver") {
        sp.advection = parse_advection(sub, context);
        sp.diffusion = parse_diffusion(sub, context);
        sp.pressure = parse_pressure(sub, context);
        sp.turbulence = parse_turbulence(sub, context);
        sp.source = parse_source(sub, context);
    } else if (d == "PressureSolver") {
        sp.pressure = parse_pressure(sub, context);
    } else {
        throw config_error("solver '" + d + "' has no parsing implementation.");
    }
    Section sol = section(sub, "solution");
    sp.analytical_solution = req_bool(sol.values, "available", ctx_join(context, "solution"));
    return sp;
}

Physical parse_physical(const XmlElement *root, const std::string &d) {
    const std::string context = "physical_parameters";
    Section s = section(root, context);
    Physical p;
    p.t_end = req_real(s.values, "t_end", context);
    p.dt = req_real(s.values, "dt", context);
    if (d != "AdvectionSolver" && d != "PressureSolver") p.nu = req_real(s.values, "nu", context);
    const bool ns = d == "NSSolver" || d == "NSTempSolver" || d == "NSTurbSolver" || d == "NSTempTurbSolver" ||
                    d == "NSTempTurbConSolver" || d == "NSTempConSolver";
    if (ns) p.rhoa = opt_real(s.values, "rhoa", 1);
    p.beta = opt_real(s.values, "beta", 3.34e-3);
    p.g = opt_real(s.values, "g", -9.81);
    if (d == "NSTempSolver" || d == "NSTempTurbSolver" || d == "NSTempTurbConSolver" || d == "NSTempConSolver")
        p.kappa = req_real(s.values, "kappa", context);
    if (d == "NSTempTurbConSolver" || d == "NSTempConSolver") p.gamma = req_real(s.values, "gamma", context);
    return p;
}

Domain parse_domain(const XmlElement *root) {
    const std::string context = "domain_parameters";
    Section s = section(root, context);
    Domain dp;
    dp.enable_computational_domain = opt_bool(s.values, "enable_computational_domain", false);
    const char *up[3] = {"X", "Y", "Z"}, *lo[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; a++) {
        dp.start_PD[a] = req_real(s.values, std::string(up[a]) + "1", context);
        dp.end_PD[a] = req_real(s.values, std::string(up[a]) + "2", context);
        dp.n[a] = req_size(s.values, std::string("n") + lo[a], context);
        if (dp.enable_computational_domain) {
            dp.start_CD[a] = req_real(s.values, std::string(lo[a]) + "1", context);
            dp.end_CD[a] = req_real(s.values, std::string(lo[a]) + "2", context);
        } else {
            dp.start_CD[a] = dp.start_PD[a];
            dp.end_CD[a] = dp.end_PD[a];
        }
    }
    return dp;
}

InitialConditions parse_ic(const XmlElement *root) {
    const std::string context = "initial_conditions";
    Section s = section(root, context);
    InitialConditions ic;
    ic.random = req_bool(s.values, "random", context);
    if (ic.random) ic.random_parameters = parse_random(need(s, context), context);
    ic.usr_fct = req_str(s.values, "usr_fct", context);
    ic.values = s.values;
    const std::string c2 = ctx_join(context, ic.usr_fct);
    // required keys per initial condition (Settings.cpp:189-331)
    static const std::map<std::string, std::vector<std::string>> required = {
        {"Uniform", {"val"}},
        {"SinSinSin", {"l"}},
        {"ExpSinusProd", {"l"}},
        {"GaussBubble", {"l", "u_lin", "v_lin", "w_lin", "x_shift", "y_shift", "z_shift"}},
        {"Hat", {"x1", "y1", "z1", "x2", "y2", "z2", "val_out", "val_in"}},
        {"Drift", {"u_lin", "v_lin", "w_lin", "pa"}},
        {"Vortex", {"u_lin", "v_lin", "w_lin", "pa", "rhoa"}},
        {"McDermott", {"A"}},
        {"Jet", {"dir", "value"}},
        {"LayersT", {"n_layers", "dir"}},
        {"Zero", {}},
        {"ExpSinusSum", {}},
    };
    auto it = required.find(ic.usr_fct);
    if (it == required.end()) throw config_error(ic.usr_fct + " has no parsing implementation.");
    // the reference reads every parameter but an axis name as a number, and a
    // value that is not one counts as missing (get_required_real, Settings.cpp:81-88)
    for (const auto &k : it->second) {
        if (k == "dir") req_str(s.values, k, c2);
        else req_real(s.values, k, c2);
    }
    if (ic.usr_fct == "Uniform") ic.uniform_value = req_real(s.values, "val", c2);
    else if (ic.usr_fct == "SinSinSin") ic.sin_l = req_real(s.values, "l", c2);
    else if (ic.usr_fct == "LayersT") {
        // parse_layers_parameters (src/utility/settings/Settings.cpp:302-321)
        const size_t n = req_size(s.values, "n_layers", c2);
        if (n == 0)
            throw config_error("Numbers of layers has to be at least 1. Current value: " + std::to_string(n));
        ic.layers_dir = match_axis(req_str(s.values, "dir", c2));
        for (size_t i = 1; i < n; i++) {
            ic.layers_values.push_back(req_real(s.values, "value_" + std::to_string(i), c2));
            ic.layers_borders.push_back(req_real(s.values, "border_" + std::to_string(i), c2));
        }
        ic.layers_values.push_back(req_real(s.values, "value_" + std::to_string(n), c2));
    }
    return ic;
}

}  // namespace

Settings parse_settings(const std::string &content, const std::string &filename) {
    std::unique_ptr<XmlElement> doc;
    try {
        doc = parse_xml(content);
    } catch (const XmlError &e) {
        throw config_error(e.what());
    }
    const XmlElement *root = doc.get();
    Settings st;
    st.filename = filename;
    st.solver = parse_solver(root);
    st.physical = parse_physical(root, st.solver.description);
    st.domain = parse_domain(root);
    {
        Section a = section(root, "adaption");
        st.adaption = req_bool(a.values, "dynamic", "adaption");
        if (st.adaption)
            throw config_error("handling of adaption is not fully implemented yet. Please check issue #178");
    }
    {
        Section b = section(root, "boundaries");
        if (b.el)
            for (const auto &c : b.el->children)
                if (c->name == "boundary") st.boundaries.push_back(parse_boundary(c.get(), "boundaries"));
    }
    {
        Section o = section(root, "obstacles");
        st.obstacles_enabled = req_bool(o.values, "enabled", "obstacles");
        if (st.obstacles_enabled) {
            for (const auto &c : o.el->children) {
                const std::string context = "obstacles/obstacle";
                Map v = attributes(c.get());
                Obstacle ob;
                ob.name = req_str(v, "name", context);
                const std::string state = opt_str(v, "state", "XML");
                if (state != "unmodified") {
                    Section g = section(c.get(), "geometry");
                    const char *lo[3] = {"x", "y", "z"};
                    for (int a = 0; a < 3; a++) {
                        ob.start[a] = req_real(g.values, std::string("o") + lo[a] + "1", context);
                        ob.end[a] = req_real(g.values, std::string("o") + lo[a] + "2", context);
                    }
                    // parse_obstacle (Settings.cpp:424-429): boundaries under "boundaries (<name>)"
                    const std::string cb = ctx_join(context, "boundaries (" + ob.name + ")");
                    for (const auto &bc : c->children)
                        if (bc->name == "boundary") ob.boundaries.push_back(parse_boundary(bc.get(), cb));
                }
                st.obstacles.push_back(ob);
            }
        }
    }
    {
        Section sf = section(root, "surfaces");
        st.surfaces_enabled = req_bool(sf.values, "enabled", "surfaces");
        if (st.surfaces_enabled && sf.el && !sf.el->children.empty())
            throw config_error("surfaces are not supported by this library (no reference configuration uses them)");
    }
    {
        // parse_assimilation_parameters (src/utility/settings/Settings.cpp:971-989).  The
        // reference acts on the section only in builds with ASSIMILATION defined (MPI
        // ranks, src/TimeIntegration.cpp:124-133 and :158-186, src/main.cpp:63-110); its serial and single-GPU
        // builds parse it and run the plain time loop.  This library does the same.
        const std::string context = "data_assimilation";
        Section da = section(root, context);
        st.assimilation.enabled = req_bool(da.values, "enabled", context);
        if (st.assimilation.enabled) {
            st.assimilation.class_name = req_str(da.values, "class_name", context);
            if (opt_bool(da.values, "load_data", false)) {
                req_str(da.values, "file", context);
                req_real(da.values, "time", context);
            }
        }
    }
    st.ic = parse_ic(root);
    {
        Section v = section(root, "visualisation");
        if (req_bool(v.values, "save_csv", "visualisation")) req_size(v.values, "csv_nth_plot", "visualisation");
        if (req_bool(v.values, "save_vtk", "visualisation")) req_size(v.values, "vtk_nth_plot", "visualisation");
    }
    {
        Section lg = section(root, "logging");
        req_str(lg.values, "file", "logging");
        req_str(lg.values, "level", "logging");
    }
    return st;
}

Settings parse_settings_file(const std::string &path) {
    std::ifstream in(path);
    if (in.fail())
        throw config_error("Could not read file '" + path +
                           "'. Please check if the file exists or the permission are sufficient.");
    std::stringstream ss;
    ss << in.rdbuf();
    std::string name = path;
    size_t slash = name.find_last_of('/');
    if (slash != std::string::npos) name = name.substr(slash + 1);
    return parse_settings(ss.str(), name);
}

}  // namespace settings
}  // namespace artss
