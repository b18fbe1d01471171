// ARTSS XML settings: the parameter tree of ARTSS src/utility/settings/Settings.h
// for the solvers this library runs, parsed with the same required/optional
// rules as Settings::parse_* (Settings.cpp:126-1053) so the same XML files are
// accepted and rejected.
#pragma once

#include <array>
#include <map>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

namespace artss {

// ARTSS enums (src/utility/Mapping.h:16-63)
enum Axis : int { AXIS_X = 0, AXIS_Y = 1, AXIS_Z = 2 };
enum PatchId : int { LEFT = 0, RIGHT = 1, BOTTOM = 2, TOP = 3, FRONT = 4, BACK = 5 };
enum FieldTypeId : int { F_RHO = 0, F_U = 1, F_V = 2, F_W = 3, F_P = 4, F_T = 5, F_NU = 6 };
enum BcType : int { BC_NEUMANN = 0, BC_DIRICHLET = 1, BC_PERIODIC = 2 };
constexpr int kPatches = 6;
constexpr int kFieldTypesHost = 7;

extern const char *const kPatchNames[kPatches];
extern const char *const kFieldTypeNames[kFieldTypesHost];

class config_error : public std::runtime_error {
 public:
    explicit config_error(const std::string &m) : std::runtime_error(m) {}
};

namespace settings {

struct Boundary {
    std::vector<int> patches;
    std::vector<int> field_types;
    int bc = BC_NEUMANN;
    std::optional<double> value;
};

struct Obstacle {
    std::string name;
    std::array<double, 3> start{}, end{};
    std::vector<Boundary> boundaries;
};

struct Domain {
    bool enable_computational_domain = false;
    std::array<double, 3> start_PD{}, end_PD{}, start_CD{}, end_CD{};
    std::array<size_t, 3> n{};
};

struct Physical {
    double t_end = 0, dt = 0;
    std::optional<double> nu, kappa, gamma, rhoa;
    double beta = 3.34e-3, g = -9.81;
};

struct Advection {
    std::string type;
    std::vector<int> fields;
};

struct Diffusion {
    std::string type;
    std::vector<int> fields;
    bool has_iteration = false;  // Jacobi / ColoredGaussSeidel
    size_t max_iter = 0;
    double tol_res = 0;
    double w = 1;
};

struct Turbulence {
    std::string type;
    bool has_cs = false;
    double cs = 0;
};

struct Source {
    std::string type;
    std::string force_fct;
    std::vector<int> dir;
    bool use_init_values = false;
    std::optional<double> ambient_temperature;
    std::array<double, 3> uniform_value{};
};

struct Pressure {
    std::string type;
    int field = F_P;
    size_t n_level = 0, n_cycle = 0, max_cycle = 0, n_relax = 0;
    double tol_res = 0;
    Diffusion smoother;
};

struct Random {
    bool absolute = false, custom_seed = false, custom_steps = false;
    size_t seed = 0;
    double step_size = 1, range = 0;
};

struct Gauss {
    double heat_release_rate = 0, heat_capacity = 1, tau = 1;
    std::array<double, 3> position{}, dimension{};
};

struct Cube {
    std::array<double, 3> start{}, end{};
    double value = 0;
};

struct TemperatureSource {
    std::string type;
    std::vector<int> dir;
    std::string temp_fct;
    bool dissipation = false;
    bool random = false;
    Random random_parameters;
    Gauss gauss;
    Cube cube;
};

struct Temperature {
    Advection advection;
    Diffusion diffusion;
    bool has_turbulence = false;
    std::optional<double> prandtl_number;
    TemperatureSource source;
};

// concentration block of NSTempConSolver / NSTempTurbConSolver
// (Settings.cpp:840-889): the source's con_fct is Gauss or Cube
struct ConcentrationSource {
    std::string type;
    std::vector<int> dir;
    std::string con_fct;
    bool random = false;
    Random random_parameters;
    Gauss gauss;
    Cube cube;
};

struct Concentration {
    Advection advection;
    Diffusion diffusion;
    bool has_turbulence = false;
    std::optional<double> turbulent_schmidt_number;
    ConcentrationSource source;
};

struct Solver {
    std::string description;
    Advection advection;
    Diffusion diffusion;
    Turbulence turbulence;
    Source source;
    Pressure pressure;
    Temperature temperature;
    Concentration concentration;
    bool analytical_solution = false;
};

struct InitialConditions {
    std::string usr_fct;
    bool random = false;
    Random random_parameters;
    double uniform_value = 0;   // Uniform: val
    double sin_l = 0;           // SinSinSin: l
    int layers_dir = -1;                  // LayersT: axis across the layers
    std::vector<double> layers_values;    // LayersT: value_1 .. value_n
    std::vector<double> layers_borders;   // LayersT: border_1 .. border_{n-1}
    std::map<std::string, std::string> values;  // all parameters of the section
};

// data_assimilation section: parsed, without effect on the time loop (as in the
// reference's builds without ASSIMILATION)
struct Assimilation {
    bool enabled = false;
    std::string class_name;
};

struct Settings {
    std::string filename;
    Physical physical;
    Solver solver;
    Domain domain;
    bool adaption = false;
    Assimilation assimilation;
    std::vector<Boundary> boundaries;
    bool obstacles_enabled = false;
    std::vector<Obstacle> obstacles;
    bool surfaces_enabled = false;
    InitialConditions ic;
};

Settings parse_settings_file(const std::string &path);
Settings parse_settings(const std::string &content, const std::string &filename);

}  // namespace settings
}  // namespace artss
