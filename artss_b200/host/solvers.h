// Field storage, solver compositions, the solver controller and the time
// loop of ARTSS (src/field/FieldController.*, src/solver/*, src/TimeIntegration.*).
#pragma once

#include <array>

#include <chrono>
#include <memory>
#include <string>
#include <vector>

#include "plugins.h"

namespace artss {

// FieldController (src/field/FieldController.h:15-137): the named fields of
// the fractional-step path, all device resident.
class FieldController {
 public:
    explicit FieldController(Runtime &rt);
    Field u, v, w, u0, v0, w0, u_tmp, v_tmp, w_tmp;
    Field nu_t, kappa_t;
    Field p, p0, rhs;
    Field T, T0, T_tmp, T_ambient;
    Field f_x, f_y, f_z;
    Field S_T;
    // concentration, its copies, source and eddy diffusivity (field type rho);
    // allocated by enable_concentration for NSTempConSolver / NSTempTurbConSolver
    std::unique_ptr<Field> C, C0, C_tmp, S_C, gamma_t;

    void enable_concentration();
    void set_up_boundary();
    void update_data();
    static void couple_vector(const Field &a, Field &a0, Field &a_tmp, const Field &b, Field &b0, Field &b_tmp,
                              const Field &c, Field &c0, Field &c_tmp);
    static void couple_scalar(const Field &a, Field &a0, Field &a_tmp);
    // a_tmp = a, b_tmp = b, c_tmp = c: the half of couple_vector that is read
    // when a0, b0, c0 are rewritten (update_data) before anything reads them
    static void couple_tmp(const Field &a, Field &a_tmp, const Field &b, Field &b_tmp, const Field &c, Field &c_tmp);
    Field *by_name(const std::string &name);

 private:
    Runtime &m_rt;
};

// ISolver (src/interfaces/ISolver.h:31-38)
class ISolver {
 public:
    virtual ~ISolver() = default;
    virtual void do_step(real t, bool sync) = 0;
    virtual void update_source(real t_cur) = 0;
    virtual void update_obstacle_change() = 0;
};

struct StepStats {
    int64_t diffusion_iterations[4] = {0, 0, 0, 0};  // u, v, w, T
    int64_t pressure_cycles = 0;
    double pressure_residual = -1;
};

// NSTempTurbSolver (src/solver/NSTempTurbSolver.cpp:94-248)
// NSTempTurbSolver (src/solver/NSTempTurbSolver.cpp); turbulent = false:
// NSTempSolver; concentration = true: NSTempTurbConSolver / NSTempConSolver
// (src/solver/NSTempTurbConSolver.cpp, NSTempConSolver.cpp)
class NSTempTurbSolver : public ISolver {
 public:
    NSTempTurbSolver(Runtime &rt, FieldController &fc, bool turbulent = true, bool concentration = false);
    void do_step(real t, bool sync) override;
    void update_source(real t_cur) override;
    void update_obstacle_change() override;
    StepStats stats;

 private:
    void couple_after_diffusion();
    Runtime &m_rt;
    FieldController &m_fc;
    bool m_turb = true;
    std::unique_ptr<IAdvection> adv_vel, adv_temp;
    std::unique_ptr<IDiffusion> dif_vel, dif_temp;
    std::unique_ptr<ITurbulence> mu_tub;
    std::unique_ptr<IPressure> pres;
    std::unique_ptr<ISource> sou_vel, sou_temp;
    std::unique_ptr<ISourceFunction> m_source_function_temperature;
    bool m_add_source = false, m_add_temp_source = false, m_dissipation = false;
    bool m_con = false, m_add_con_source = false;
    std::unique_ptr<IAdvection> adv_con;
    std::unique_ptr<IDiffusion> dif_con;
    std::unique_ptr<ISource> sou_con;
    std::unique_ptr<ISourceFunction> m_source_function_concentration;
};

// NSSolver / NSTurbSolver (src/solver/NSSolver.cpp, NSTurbSolver.cpp)
class NSSolver : public ISolver {
 public:
    NSSolver(Runtime &rt, FieldController &fc, bool turbulent);
    void do_step(real t, bool sync) override;
    void update_source(real) override {}
    void update_obstacle_change() override {}

 private:
    Runtime &m_rt;
    FieldController &m_fc;
    bool m_turb;
    std::unique_ptr<IAdvection> adv_vel;
    std::unique_ptr<IDiffusion> dif_vel;
    std::unique_ptr<ITurbulence> mu_tub;
    std::unique_ptr<IPressure> pres;
    std::unique_ptr<ISource> sou_vel;
    bool m_add_source = false;
};

// AdvectionSolver, AdvectionDiffusionSolver, DiffusionSolver, DiffusionTurbSolver
// (src/solver/AdvectionSolver.cpp, AdvectionDiffusionSolver.cpp, DiffusionSolver.cpp,
// DiffusionTurbSolver.cpp): the velocity-only compositions of the same plugins.
class VelocitySolver : public ISolver {
 public:
    enum Kind { ADVECTION, ADVECTION_DIFFUSION, DIFFUSION, DIFFUSION_TURB };
    VelocitySolver(Runtime &rt, FieldController &fc, Kind kind, std::array<real, 3> velocity_lin = {0, 0, 0});
    void do_step(real t, bool sync) override;
    void update_source(real) override {}
    void update_obstacle_change() override {}

 private:
    Runtime &m_rt;
    FieldController &m_fc;
    Kind m_kind;
    std::unique_ptr<IAdvection> adv;
    std::unique_ptr<IDiffusion> dif;
    std::unique_ptr<ITurbulence> mu_tub;
    std::unique_ptr<Field> m_u_lin, m_v_lin, m_w_lin;  // AdvectionSolver's constant transport velocity
};

// PressureSolver (src/solver/PressureSolver.cpp:30-43)
class PressureSolver : public ISolver {
 public:
    PressureSolver(Runtime &rt, FieldController &fc);
    void do_step(real t, bool sync) override;
    void update_source(real) override {}
    void update_obstacle_change() override {}
    IPressure &pressure() { return *pres; }

 private:
    FieldController &m_fc;
    std::unique_ptr<IPressure> pres;
};

// SolverController (src/solver/SolverController.cpp:26-311)
class SolverController {
 public:
    SolverController(Runtime &rt);
    void solver_do_step(real t, bool sync) { m_solver->do_step(t, sync); }
    void update_sources(real t_cur, bool sync);
    FieldController &fields() { return *m_fc; }
    ISolver &solver() { return *m_solver; }

 private:
    void set_up_fields();
    void force_source();
    void momentum_source();
    Runtime &m_rt;
    std::unique_ptr<FieldController> m_fc;
    std::unique_ptr<ISolver> m_solver;
    bool m_has_momentum_source = false;
};

// TimeIntegration (src/TimeIntegration.cpp:45-186), benchmark branch.
class TimeIntegration {
 public:
    TimeIntegration(Runtime &rt, SolverController &sc);
    ~TimeIntegration();
    TimeIntegration(const TimeIntegration &) = delete;
    TimeIntegration &operator=(const TimeIntegration &) = delete;
    // runs until t_end (steps < 0) or for `steps` steps; returns steps run
    int64_t run(int64_t steps = -1);
    // one step with its host transfers: the inputs are uploaded into their
    // fields, the outputs read back, overlapped with the step where the
    // solver marks first uses and final writes (StepIO); the transfers are
    // complete when the context's stream reaches them
    void step_io(const std::vector<std::pair<Field *, const real *>> &in,
                 const std::vector<std::pair<Field *, real *>> &out);
    // the step with pipelined transfers (artss_io_in / artss_io_out): returns
    // once they and the step are enqueued
    void step_io_async(const std::vector<std::pair<Field *, const real *>> &in,
                       const std::vector<std::pair<Field *, real *>> &out);
    real time() const { return m_t_cur; }
    int64_t step_index() const { return m_step; }
    bool finished() const;
    // continue from step `step` (its time is step * dt), e.g. after a rollback
    void set_step(int64_t step);

 private:
    // the step as one graph (Runtime::graphs): captured at step kGraphStep,
    // replayed after; a step that cannot be captured keeps the eager path
    void capture_step();
    static constexpr int64_t kGraphStep = 3;
    artss_graph *m_graph = nullptr;
    bool m_graph_failed = false;

 public:
    int64_t graph_steps = 0;  // steps run as a graph launch

 private:

    Runtime &m_rt;
    SolverController &m_sc;
    real m_dt, m_t_end, m_t_cur;
    int64_t m_step = 1;
};

// Plugin factory of src/solver/SolverSelection.cpp:33-212.
std::unique_ptr<IAdvection> make_advection(Runtime &rt, const settings::Advection &s);
std::unique_ptr<IDiffusion> make_diffusion(Runtime &rt, const settings::Diffusion &s);
std::unique_ptr<ITurbulence> make_turbulence(Runtime &rt, const settings::Turbulence &s);
std::unique_ptr<IPressure> make_pressure(Runtime &rt, const settings::Pressure &s);
std::unique_ptr<ISource> make_source(Runtime &rt, const std::string &type, const std::vector<int> &dir);

}  // namespace artss
