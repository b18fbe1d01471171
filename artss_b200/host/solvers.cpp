#include "solvers.h"

#include <algorithm>
#include <cmath>

namespace artss {

// ---------------------------------------------------------------- factory

std::unique_ptr<IAdvection> make_advection(Runtime &rt, const settings::Advection &s) {
    if (s.type == "SemiLagrangian") return std::make_unique<SLAdvect>(rt);
    throw config_error("advection method '" + s.type + "' is not implemented");
}

std::unique_ptr<IDiffusion> make_diffusion(Runtime &rt, const settings::Diffusion &s) {
    if (s.type == "ColoredGaussSeidel") return std::make_unique<ColoredGaussSeidelDiffuse>(rt, s);
    if (s.type == "ColoredGaussSeidelMixed") return std::make_unique<ColoredGaussSeidelDiffuse>(rt, s, true);
    if (s.type == "Jacobi") return std::make_unique<JacobiDiffuse>(rt, s);
    if (s.type == "Explicit") return std::make_unique<ExplicitDiffuse>(rt);
    throw config_error("diffusion method '" + s.type + "' is not implemented");
}

std::unique_ptr<ITurbulence> make_turbulence(Runtime &rt, const settings::Turbulence &s) {
    if (s.type == "ConstSmagorinsky") return std::make_unique<ConstSmagorinsky>(rt, s.cs);
    if (s.type == "DynamicSmagorinsky") return std::make_unique<DynamicSmagorinsky>(rt);
    throw config_error("turbulence method '" + s.type + "' is not implemented");
}

std::unique_ptr<IPressure> make_pressure(Runtime &rt, const settings::Pressure &s) {
    if (s.type == "VCycleMG") return std::make_unique<VCycleMG>(rt, s);
    if (s.type == "VCycleMGRel") return std::make_unique<VCycleMG>(rt, s, true);
    if (s.type == "VCycleMGMixed") return std::make_unique<MixedVCycle>(rt, s);
    throw config_error("pressure method '" + s.type + "' is not implemented");
}

std::unique_ptr<ISource> make_source(Runtime &rt, const std::string &type, const std::vector<int> &dir) {
    if (type == "ExplicitEuler") return std::make_unique<ExplicitEulerSource>(rt, dir);
    throw config_error("source method '" + type + "' is not implemented");
}

static std::unique_ptr<ISourceFunction> make_temperature_source_function(Runtime &rt,
                                                                          const settings::TemperatureSource &s) {
    // SolverSelection::set_temperature_source_function (src/solver/SolverSelection.cpp:138-163)
    if (s.temp_fct == "Gauss") {
        auto g = std::make_unique<GaussFunction>(rt, s.gauss);
        if (s.random) {
            const auto &r = s.random_parameters;
            if (!r.custom_seed)
                throw config_error("a temperature-source noise without custom_seed is not reproducible");
            g->set_noise(std::make_unique<UniformRandom>(r.range, r.step_size, r.seed), r.absolute);
        }
        return g;
    }
    if (s.temp_fct == "Zero") return std::make_unique<ZeroSource>();
    throw config_error("temperature source function '" + s.temp_fct + "' is not implemented");
}

// SolverSelection::set_concentration_source_function (src/solver/SolverSelection.cpp:165-190):
// the Gauss function of the concentration settings
static std::unique_ptr<ISourceFunction> make_concentration_source_function(Runtime &rt,
                                                                            const settings::ConcentrationSource &s) {
    if (s.con_fct == "Gauss") {
        if (s.random) throw config_error("a concentration-source noise is not implemented");
        return std::make_unique<GaussFunction>(rt, s.gauss);
    }
    throw config_error("concentration source function '" + s.con_fct + "' is not implemented");
}

// ---------------------------------------------------------------- fields

FieldController::FieldController(Runtime &rt)
    : u(rt, F_U), v(rt, F_V), w(rt, F_W), u0(rt, F_U), v0(rt, F_V), w0(rt, F_W), u_tmp(rt, F_U), v_tmp(rt, F_V),
      w_tmp(rt, F_W), nu_t(rt, F_NU), kappa_t(rt, F_T), p(rt, F_P), p0(rt, F_P), rhs(rt, F_P), T(rt, F_T),
      T0(rt, F_T), T_tmp(rt, F_T), T_ambient(rt, F_T), f_x(rt, F_U), f_y(rt, F_V), f_z(rt, F_W), S_T(rt, F_T),
      m_rt(rt) {}

void FieldController::enable_concentration() {
    if (C) return;
    C = std::make_unique<Field>(m_rt, F_RHO);
    C0 = std::make_unique<Field>(m_rt, F_RHO);
    C_tmp = std::make_unique<Field>(m_rt, F_RHO);
    S_C = std::make_unique<Field>(m_rt, F_RHO);
    gamma_t = std::make_unique<Field>(m_rt, F_RHO);
}

void FieldController::set_up_boundary() {
    // FieldController::set_up_boundary (src/field/FieldController.cpp:102-112); without a
    // concentration solver the concentration field is all zero and unused here
    m_rt.apply_boundary(u);
    m_rt.apply_boundary(v);
    m_rt.apply_boundary(w);
    m_rt.apply_boundary(p);
    m_rt.apply_boundary(T);
    if (C) m_rt.apply_boundary(*C);
    m_rt.apply_boundary(T_ambient);
}

void FieldController::update_data() {
    // FieldController::update_data (src/field/FieldController.cpp:119-135)
    couple_vector(u, u0, u_tmp, v, v0, v_tmp, w, w0, w_tmp);
    p0.copy_data(p);
    couple_scalar(T, T0, T_tmp);
    if (C) couple_scalar(*C, *C0, *C_tmp);
}

void FieldController::couple_vector(const Field &a, Field &a0, Field &a_tmp, const Field &b, Field &b0, Field &b_tmp,
                                    const Field &c, Field &c0, Field &c_tmp) {
    check(artss_couple(a.runtime().ctx(), a.data, a0.data, a_tmp.data, b.data, b0.data, b_tmp.data, c.data, c0.data,
                       c_tmp.data),
          "couple_vector");
}

void FieldController::couple_tmp(const Field &a, Field &a_tmp, const Field &b, Field &b_tmp, const Field &c,
                                 Field &c_tmp) {
    check(artss_couple(a.runtime().ctx(), a.data, nullptr, a_tmp.data, b.data, nullptr, b_tmp.data, c.data, nullptr,
                       c_tmp.data),
          "couple_tmp");
}

void FieldController::couple_scalar(const Field &a, Field &a0, Field &a_tmp) {
    check(artss_couple(a.runtime().ctx(), a.data, a0.data, a_tmp.data, nullptr, nullptr, nullptr, nullptr, nullptr,
                       nullptr),
          "couple_scalar");
}

Field *FieldController::by_name(const std::string &n) {
    if (n == "u") return &u;
    if (n == "v") return &v;
    if (n == "w") return &w;
    if (n == "u0") return &u0;
    if (n == "v0") return &v0;
    if (n == "w0") return &w0;
    if (n == "u_tmp") return &u_tmp;
    if (n == "v_tmp") return &v_tmp;
    if (n == "w_tmp") return &w_tmp;
    if (n == "nu_t") return &nu_t;
    if (n == "kappa_t") return &kappa_t;
    if (n == "p") return &p;
    if (n == "p0") return &p0;
    if (n == "rhs") return &rhs;
    if (n == "T") return &T;
    if (n == "T0") return &T0;
    if (n == "T_tmp") return &T_tmp;
    if (n == "T_a") return &T_ambient;
    if (n == "f_x") return &f_x;
    if (n == "f_y") return &f_y;
    if (n == "f_z") return &f_z;
    if (n == "S_T") return &S_T;
    if (n == "C") return C.get();
    if (n == "C0") return C0.get();
    if (n == "C_tmp") return C_tmp.get();
    if (n == "S_C") return S_C.get();
    if (n == "gamma_t") return gamma_t.get();
    return nullptr;
}

// ---------------------------------------------------------------- NSTempTurbSolver

NSTempTurbSolver::NSTempTurbSolver(Runtime &rt, FieldController &fc, bool turbulent, bool concentration)
    : m_rt(rt), m_fc(fc), m_turb(turbulent), m_con(concentration) {
    // NSTempSolver (src/solver/NSTempSolver.cpp:16-49) is the same composition
    // without the turbulence model
    const settings::Solver &s = rt.settings().solver;
    adv_vel = make_advection(rt, s.advection);
    adv_temp = make_advection(rt, s.temperature.advection);
    dif_vel = make_diffusion(rt, s.diffusion);
    if (turbulent) mu_tub = make_turbulence(rt, s.turbulence);
    dif_temp = make_diffusion(rt, s.diffusion);  // NSTempTurbSolver.cpp:50: the velocity settings
    pres = make_pressure(rt, s.pressure);
    sou_vel = make_source(rt, s.source.type, s.source.dir);
    sou_temp = make_source(rt, s.temperature.source.type, s.temperature.source.dir);
    m_source_function_temperature = make_temperature_source_function(rt, s.temperature.source);
    m_add_source = s.source.force_fct != "Zero";
    m_add_temp_source = s.temperature.source.temp_fct != "Zero";
    // NSTempTurbSolver::control (:254-298)
    auto sorted = [](std::vector<int> v) { std::sort(v.begin(), v.end()); return v; };
    if (sorted(s.advection.fields) != std::vector<int>{F_U, F_V, F_W} ||
        sorted(s.diffusion.fields) != std::vector<int>{F_U, F_V, F_W} ||
        s.temperature.advection.fields != std::vector<int>{F_T} ||
        s.temperature.diffusion.fields != std::vector<int>{F_T} || s.pressure.field != F_P)
        throw config_error("Fields not specified correctly!");
    m_dissipation = s.temperature.source.dissipation;
    // `in` of every diffuse() call below is re-coupled before it is read again,
    // and out and in are coupled from one field just before each call
    dif_vel->in_is_scratch = true;
    dif_temp->in_is_scratch = true;
    dif_vel->out_holds_in = true;
    dif_temp->out_holds_in = true;
    if (m_con) {
        // NSTempTurbConSolver.cpp:28-53 / NSTempConSolver.cpp:29-51, with the concentration's
        // advection held in its own slot (the reference stores it in adv_temp a second time
        // and never sets adv_con, so its do_step cannot run; this is the evident intent)
        m_fc.enable_concentration();
        adv_con = make_advection(rt, s.concentration.advection);
        dif_con = make_diffusion(rt, s.diffusion);  // the velocity settings, as for the temperature
        sou_con = make_source(rt, s.concentration.source.type, s.concentration.source.dir);
        m_source_function_concentration = make_concentration_source_function(rt, s.concentration.source);
        m_add_con_source = s.concentration.source.con_fct != "Zero";
        if (s.concentration.advection.fields != std::vector<int>{F_RHO} ||
            s.concentration.diffusion.fields != std::vector<int>{F_RHO})
            throw config_error("Fields not specified correctly!");
        if (!m_rt.settings().physical.gamma) throw config_error("physical_parameters: gamma missing");
    }
}

void NSTempTurbSolver::do_step(real t, bool sync) {
    FieldController &f = m_fc;
    const auto &phys = m_rt.settings().physical;
    const real nu = phys.nu.value();
    const real kappa = phys.kappa.value();
    artss_ctx *ctx = m_rt.ctx();

    // 1. advection of velocity with the old velocity (:129-131)
    artss_ctx_stage_mark(ctx, ARTSS_STAGE_ADVECTION);
    if (auto *sl = dynamic_cast<SLAdvect *>(adv_vel.get())) {
        sl->advect_vector(f.u, f.v, f.w, f.u0, f.v0, f.w0, f.u0, f.v0, f.w0);
    } else {
        adv_vel->advect(f.u, f.u0, f.u0, f.v0, f.w0, sync);
        adv_vel->advect(f.v, f.v0, f.u0, f.v0, f.w0, sync);
        adv_vel->advect(f.w, f.w0, f.u0, f.v0, f.w0, sync);
    }
    FieldController::couple_vector(f.u, f.u0, f.u_tmp, f.v, f.v0, f.v_tmp, f.w, f.w0, f.w_tmp);

    // 2. turbulent viscosity and diffusion (:140-152); NSTempSolver: laminar
    //    diffusion when nu != 0 (NSTempSolver.cpp:109-119)
    artss_ctx_stage_mark(ctx, ARTSS_STAGE_DIFFUSION);
    if (m_turb) {
        mu_tub->calc_turbulent_viscosity(f.nu_t, f.u, f.v, f.w, true);
        dif_vel->diffuse(f.u, f.u0, f.u_tmp, nu, f.nu_t, sync);
        stats.diffusion_iterations[0] = dif_vel->last_iterations;
        dif_vel->diffuse(f.v, f.v0, f.v_tmp, nu, f.nu_t, sync);
        stats.diffusion_iterations[1] = dif_vel->last_iterations;
        dif_vel->diffuse(f.w, f.w0, f.w_tmp, nu, f.nu_t, sync);
        stats.diffusion_iterations[2] = dif_vel->last_iterations;
        couple_after_diffusion();
    } else if (nu != 0.) {
        dif_vel->diffuse(f.u, f.u0, f.u_tmp, nu, sync);
        stats.diffusion_iterations[0] = dif_vel->last_iterations;
        dif_vel->diffuse(f.v, f.v0, f.v_tmp, nu, sync);
        stats.diffusion_iterations[1] = dif_vel->last_iterations;
        dif_vel->diffuse(f.w, f.w0, f.w_tmp, nu, sync);
        stats.diffusion_iterations[2] = dif_vel->last_iterations;
        couple_after_diffusion();
    }

    // 3. momentum source (:155-163); its couple_vector (:162) writes u0, v0, w0 that
    //    update_data rewrites before they are read: the u_tmp half only
    artss_ctx_stage_mark(ctx, ARTSS_STAGE_SOURCE);
    if (m_add_source) {
        sou_vel->add_source(f.u, f.v, f.w, f.f_x, f.f_y, f.f_z, sync);
        FieldController::couple_tmp(f.u, f.u_tmp, f.v, f.v_tmp, f.w, f.w_tmp);
    }

    // 4. pressure and projection (:167-176)
    artss_ctx_stage_mark(ctx, ARTSS_STAGE_PRESSURE);
    pres->divergence(f.rhs, f.u_tmp, f.v_tmp, f.w_tmp, sync);
    if (m_rt.io) m_rt.io->need(f.p);
    pres->pressure(f.p, f.rhs, t, sync);
    stats.pressure_cycles = pres->last_cycles;
    stats.pressure_residual = pres->last_residual;
    pres->projection(f.u, f.v, f.w, f.u_tmp, f.v_tmp, f.w_tmp, f.p, sync);
    if (m_rt.io) {
        // u, v, w and p are final for this step; an uploaded T is the state
        // the temperature step advances (its copies follow, as after a step)
        for (Field *x : {&f.u, &f.v, &f.w, &f.p}) m_rt.io->done(*x);
        if (m_rt.io->need(f.T)) FieldController::couple_scalar(f.T, f.T0, f.T_tmp);
    }

    // 5. temperature (:184-240)
    artss_ctx_stage_mark(ctx, ARTSS_STAGE_TEMPERATURE);
    adv_temp->advect(f.T, f.T0, f.u, f.v, f.w, sync);
    FieldController::couple_scalar(f.T, f.T0, f.T_tmp);
    const auto &ts = m_rt.settings().solver.temperature;
    // The couple_scalar calls that follow the temperature's diffusion and source
    // (:206, :216, :239) are left out: the source reads T and S_T only, and
    // nothing reads T0 or T_tmp before update_data couples T again at the end
    // of the step (TimeIntegration::run), so the fields after the step are the same.
    if (m_turb && ts.has_turbulence) {
        const real rPr_T = 1. / ts.prandtl_number.value();
        check(artss_scale_copy(m_rt.ctx(), f.kappa_t.data, f.nu_t.data, rPr_T, 0), "kappa_t");
        dif_temp->diffuse(f.T, f.T0, f.T_tmp, kappa, f.kappa_t, sync);
        stats.diffusion_iterations[3] = dif_temp->last_iterations;
    } else if (kappa != 0.) {
        dif_temp->diffuse(f.T, f.T0, f.T_tmp, kappa, sync);
        stats.diffusion_iterations[3] = dif_temp->last_iterations;
    }
    // dissipation then the source (NSTempTurbSolver.cpp:220-240, NSTempSolver.cpp:168-190); the couple
    // after each writes T0 and T_tmp, which update_data rewrites before anything reads them
    if (m_dissipation) sou_temp->dissipate(f.T, f.u, f.v, f.w, sync);
    if (m_add_temp_source) sou_temp->add_source(f.T, f.S_T, sync);

    // 6. concentration (NSTempTurbConSolver.cpp:243-286, NSTempConSolver.cpp:203-232)
    if (!m_con) return;
    Field &C = *f.C, &C0 = *f.C0, &C_tmp = *f.C_tmp;
    const real gamma = phys.gamma.value();
    const auto &cs = m_rt.settings().solver.concentration;
    adv_con->advect(C, C0, f.u, f.v, f.w, sync);
    FieldController::couple_scalar(C, C0, C_tmp);
    if (m_turb && cs.has_turbulence) {
        const real rSc_T = 1. / cs.turbulent_schmidt_number.value();
        check(artss_scale_copy(m_rt.ctx(), f.gamma_t->data, f.nu_t.data, rSc_T, 0), "gamma_t");
        dif_con->diffuse(C, C0, C_tmp, gamma, *f.gamma_t, sync);
        FieldController::couple_scalar(C, C0, C_tmp);
    } else if (gamma != 0.) {
        dif_con->diffuse(C, C0, C_tmp, gamma, sync);
        FieldController::couple_scalar(C, C0, C_tmp);
    }
    // the turbulent solver adds the source when the concentration has turbulence
    // (NSTempTurbConSolver.cpp:278), the laminar one when a source function is set
    if (m_turb ? cs.has_turbulence : m_add_con_source) {
        sou_con->add_source(C, *f.S_C, sync);
        FieldController::couple_scalar(C, C0, C_tmp);
    }
}

// couple_vector after the velocity diffusion (:152): with a momentum source
// next, which reads u, v, w and the forces only and is followed by its own
// couple, it is left out; otherwise the divergence reads u_tmp, v_tmp, w_tmp
// and u0, v0, w0 are rewritten by update_data before they are read.
void NSTempTurbSolver::couple_after_diffusion() {
    FieldController &f = m_fc;
    if (!m_add_source) FieldController::couple_tmp(f.u, f.u_tmp, f.v, f.v_tmp, f.w, f.w_tmp);
}

void NSTempTurbSolver::update_source(real t_cur) {
    m_source_function_temperature->update_source(m_fc.S_T, t_cur);
    if (m_con) m_source_function_concentration->update_source(*m_fc.S_C, t_cur);
}

void NSTempTurbSolver::update_obstacle_change() {
    m_source_function_temperature->update_obstacle_change();
    if (m_con) m_source_function_concentration->update_obstacle_change();
}

// ---------------------------------------------------------------- NSSolver / NSTurbSolver

NSSolver::NSSolver(Runtime &rt, FieldController &fc, bool turbulent) : m_rt(rt), m_fc(fc), m_turb(turbulent) {
    const settings::Solver &s = rt.settings().solver;
    adv_vel = make_advection(rt, s.advection);
    dif_vel = make_diffusion(rt, s.diffusion);
    if (turbulent) mu_tub = make_turbulence(rt, s.turbulence);
    pres = make_pressure(rt, s.pressure);
    sou_vel = make_source(rt, s.source.type, s.source.dir);
    m_add_source = s.source.force_fct != "Zero";
    dif_vel->in_is_scratch = true;
}

void NSSolver::do_step(real t, bool sync) {
    FieldController &f = m_fc;
    const real nu = m_rt.settings().physical.nu.value();
    if (auto *sl = dynamic_cast<SLAdvect *>(adv_vel.get())) {
        sl->advect_vector(f.u, f.v, f.w, f.u0, f.v0, f.w0, f.u0, f.v0, f.w0);
    } else {
        adv_vel->advect(f.u, f.u0, f.u0, f.v0, f.w0, sync);
        adv_vel->advect(f.v, f.v0, f.u0, f.v0, f.w0, sync);
        adv_vel->advect(f.w, f.w0, f.u0, f.v0, f.w0, sync);
    }
    FieldController::couple_vector(f.u, f.u0, f.u_tmp, f.v, f.v0, f.v_tmp, f.w, f.w0, f.w_tmp);
    if (m_turb) {
        // NSTurbSolver.cpp: turbulent viscosity, then turbulent diffusion
        mu_tub->calc_turbulent_viscosity(f.nu_t, f.u, f.v, f.w, true);
        dif_vel->diffuse(f.u, f.u0, f.u_tmp, nu, f.nu_t, sync);
        dif_vel->diffuse(f.v, f.v0, f.v_tmp, nu, f.nu_t, sync);
        dif_vel->diffuse(f.w, f.w0, f.w_tmp, nu, f.nu_t, sync);
        FieldController::couple_vector(f.u, f.u0, f.u_tmp, f.v, f.v0, f.v_tmp, f.w, f.w0, f.w_tmp);
    } else if (nu != 0.) {
        dif_vel->diffuse(f.u, f.u0, f.u_tmp, nu, sync);
        dif_vel->diffuse(f.v, f.v0, f.v_tmp, nu, sync);
        dif_vel->diffuse(f.w, f.w0, f.w_tmp, nu, sync);
        FieldController::couple_vector(f.u, f.u0, f.u_tmp, f.v, f.v0, f.v_tmp, f.w, f.w0, f.w_tmp);
    }
    if (m_add_source) {
        sou_vel->add_source(f.u, f.v, f.w, f.f_x, f.f_y, f.f_z, sync);
        FieldController::couple_vector(f.u, f.u0, f.u_tmp, f.v, f.v0, f.v_tmp, f.w, f.w0, f.w_tmp);
    }
    pres->divergence(f.rhs, f.u_tmp, f.v_tmp, f.w_tmp, sync);
    pres->pressure(f.p, f.rhs, t, sync);
    pres->projection(f.u, f.v, f.w, f.u_tmp, f.v_tmp, f.w_tmp, f.p, sync);
}

// ---------------------------------------------------------------- velocity-only solvers

VelocitySolver::VelocitySolver(Runtime &rt, FieldController &fc, Kind kind, std::array<real, 3> velocity_lin)
    : m_rt(rt), m_fc(fc), m_kind(kind) {
    const settings::Solver &s = rt.settings().solver;
    if (kind == ADVECTION || kind == ADVECTION_DIFFUSION) adv = make_advection(rt, s.advection);
    if (kind != ADVECTION) dif = make_diffusion(rt, s.diffusion);
    if (kind == DIFFUSION_TURB) mu_tub = make_turbulence(rt, s.turbulence);
    if (kind == ADVECTION) {
        // AdvectionSolver.cpp:17-27: constant fields of the GaussBubble velocity
        m_u_lin = std::make_unique<Field>(rt, F_U, velocity_lin[0]);
        m_v_lin = std::make_unique<Field>(rt, F_V, velocity_lin[1]);
        m_w_lin = std::make_unique<Field>(rt, F_W, velocity_lin[2]);
    }
}

void VelocitySolver::do_step(real, bool sync) {
    FieldController &f = m_fc;
    const real nu = m_rt.settings().physical.nu.value_or(0.0);
    switch (m_kind) {
        case ADVECTION:  // AdvectionSolver.cpp:57-79
            adv->advect(f.u, f.u0, *m_u_lin, *m_v_lin, *m_w_lin, sync);
            adv->advect(f.v, f.v0, *m_u_lin, *m_v_lin, *m_w_lin, sync);
            adv->advect(f.w, f.w0, *m_u_lin, *m_v_lin, *m_w_lin, sync);
            break;
        case ADVECTION_DIFFUSION:  // AdvectionDiffusionSolver.cpp:42-84
            adv->advect(f.u, f.u0, f.u0, f.v0, f.w0, sync);
            adv->advect(f.v, f.v0, f.u0, f.v0, f.w0, sync);
            adv->advect(f.w, f.w0, f.u0, f.v0, f.w0, sync);
            FieldController::couple_vector(f.u, f.u0, f.u_tmp, f.v, f.v0, f.v_tmp, f.w, f.w0, f.w_tmp);
            if (nu != 0.) {
                dif->diffuse(f.u, f.u0, f.u_tmp, nu, sync);
                dif->diffuse(f.v, f.v0, f.v_tmp, nu, sync);
                dif->diffuse(f.w, f.w0, f.w_tmp, nu, sync);
            }
            break;
        case DIFFUSION:  // DiffusionSolver.cpp:39-65
            dif->diffuse(f.u, f.u0, f.u_tmp, nu, sync);
            dif->diffuse(f.v, f.v0, f.v_tmp, nu, sync);
            dif->diffuse(f.w, f.w0, f.w_tmp, nu, sync);
            break;
        case DIFFUSION_TURB:  // DiffusionTurbSolver.cpp:38-68
            mu_tub->calc_turbulent_viscosity(f.nu_t, f.u, f.v, f.w, true);
            dif->diffuse(f.u, f.u0, f.u_tmp, nu, f.nu_t, sync);
            dif->diffuse(f.v, f.v0, f.v_tmp, nu, f.nu_t, sync);
            dif->diffuse(f.w, f.w0, f.w_tmp, nu, f.nu_t, sync);
            break;
    }
}

// ---------------------------------------------------------------- PressureSolver

PressureSolver::PressureSolver(Runtime &rt, FieldController &fc) : m_fc(fc) {
    if (rt.settings().solver.pressure.field != F_P) throw config_error("Fields not specified correctly!");
    pres = make_pressure(rt, rt.settings().solver.pressure);
}

void PressureSolver::do_step(real t, bool sync) { pres->pressure(m_fc.p, m_fc.rhs, t, sync); }

// ---------------------------------------------------------------- SolverController

SolverController::SolverController(Runtime &rt) : m_rt(rt) {
    m_fc = std::make_unique<FieldController>(rt);
    const std::string &d = rt.settings().solver.description;
    if (d == "NSTempTurbSolver" || d == "NSTempSolver" || d == "NSTempTurbConSolver" || d == "NSTempConSolver") {
        m_solver = std::make_unique<NSTempTurbSolver>(rt, *m_fc, d == "NSTempTurbSolver" || d == "NSTempTurbConSolver",
                                                      d == "NSTempTurbConSolver" || d == "NSTempConSolver");
        m_has_momentum_source = true;
    } else if (d == "NSSolver" || d == "NSTurbSolver") {
        m_solver = std::make_unique<NSSolver>(rt, *m_fc, d == "NSTurbSolver");
        m_has_momentum_source = true;
    } else if (d == "PressureSolver") {
        m_solver = std::make_unique<PressureSolver>(rt, *m_fc);
    } else if (d == "AdvectionSolver") {
        // SolverController.cpp:54-56: the transport velocity is the GaussBubble's
        const auto &v = rt.settings().ic.values;
        if (rt.settings().ic.usr_fct != "GaussBubble")
            throw config_error("AdvectionSolver takes its velocity from the GaussBubble initial condition");
        m_solver = std::make_unique<VelocitySolver>(
            rt, *m_fc, VelocitySolver::ADVECTION,
            std::array<real, 3>{std::stod(v.at("u_lin")), std::stod(v.at("v_lin")), std::stod(v.at("w_lin"))});
    } else if (d == "AdvectionDiffusionSolver") {
        m_solver = std::make_unique<VelocitySolver>(rt, *m_fc, VelocitySolver::ADVECTION_DIFFUSION);
    } else if (d == "DiffusionSolver") {
        m_solver = std::make_unique<VelocitySolver>(rt, *m_fc, VelocitySolver::DIFFUSION);
    } else if (d == "DiffusionTurbSolver") {
        m_solver = std::make_unique<VelocitySolver>(rt, *m_fc, VelocitySolver::DIFFUSION_TURB);
    } else {
        throw config_error("Solver " + d + " not yet implemented on this path");
    }
    set_up_fields();
    m_fc->set_up_boundary();
    update_sources(0, true);
    m_fc->update_data();
}

void SolverController::set_up_fields() {
    // SolverController::set_up_fields (src/solver/SolverController.cpp:95-205), the
    // initial conditions of the fractional-step path
    const auto &ic = m_rt.settings().ic;
    const Geometry &geo = m_rt.geometry();
    const IdxList &inner = geo.inner(0);
    auto add_random = [&](std::vector<real> &T) {
        // Functions::random (src/Functions.cpp:738-774); the draws cover
        // all Nx*Ny*Nz cells in linear order, applied to inner cells
        if (!ic.random) return;
        const auto &r = ic.random_parameters;
        if (!r.custom_seed) throw config_error("initial noise without custom_seed is not reproducible");
        if (!r.absolute && (r.range > 1 || r.range < 0))
            throw config_error("range for relative noise has to be between [0:1]");
        UniformRandom noise(r.range, r.step_size, r.seed);
        std::vector<real> n = noise.random_field(T.size());
        for (Idx idx : inner) {
            if (r.absolute) T[(size_t) idx] += n[(size_t) idx];
            else T[(size_t) idx] *= (1 + n[(size_t) idx]);
        }
    };
    if (ic.usr_fct == "Uniform") {
        std::vector<real> T = m_fc->T.to_host();
        for (Idx idx : inner) T[(size_t) idx] = ic.uniform_value;
        add_random(T);
        m_fc->T.from_host(T);
    } else if (ic.usr_fct == "LayersT") {
        // Functions::layers (src/Functions.cpp:521-594): layer l covers the cells whose
        // lower face lies in [border_l, border_{l+1}], the outer borders being the
        // computational domain's; layers are written in order, so a cell whose face
        // sits on a border takes the upper layer's value
        std::vector<real> T = m_fc->T.to_host();
        const int dir = ic.layers_dir;
        // an axis name the reference does not know fails its first coordinate
        // lookup (Coordinate::operator[], src/domain/Coordinate.h:53)
        if (dir < 0) throw config_error("unknown axis");
        {
            const Grid &grid = geo.grid();
            const GridLevel &g = grid.level(0);
            const size_t n = ic.layers_values.size();
            std::vector<real> borders(n + 1);
            for (size_t l = 1; l < n; l++) borders[l] = ic.layers_borders[l - 1];
            borders[0] = grid.start_cd[dir];
            borders[n] = grid.end_cd[dir];
            const size_t Nx = g.N[0], Nxy = g.N[0] * g.N[1];
            const real X1 = grid.start_pd[dir], h = g.spacing[dir];
            for (size_t l = 0; l < n; l++)
                for (Idx idx : inner) {
                    const size_t k = (size_t) idx / Nxy, j = ((size_t) idx - k * Nxy) / Nx;
                    const size_t i = (size_t) idx - k * Nxy - j * Nx;
                    const size_t c = dir == 0 ? i : dir == 1 ? j : k;
                    const real x = (X1 + ((real) c - 0.5) * h) - 0.5 * h;
                    if (borders[l] <= x && x <= borders[l + 1]) T[(size_t) idx] = ic.layers_values[l];
                }
        }
        add_random(T);
        m_fc->T.from_host(T);
    } else if (ic.usr_fct == "ExpSinusSum") {
        // Functions::exp_sinus_sum (src/Functions.cpp:369-420) at t = 0: the Burgers
        // test state on the inner cells of u, v and w, 3D when Nz > 3
        const GridLevel &g = geo.grid().level(0);
        const auto &X1 = geo.grid().start_pd;
        const size_t Nx = g.N[0], Nxy = g.N[0] * g.N[1];
        const real nu = m_rt.settings().physical.nu.value_or(0.0), t = 0.;
        const bool three_d = g.N[2] > 3;
        const real d = three_d ? 3. : 2.;
        std::vector<real> u = m_fc->u.to_host(), v = m_fc->v.to_host(), w = m_fc->w.to_host();
        for (Idx idx : inner) {
            const size_t k = (size_t) idx / Nxy, j = ((size_t) idx - k * Nxy) / Nx, i = (size_t) idx - k * Nxy - j * Nx;
            const real xi = X1[0] + ((real) i - 0.5) * g.spacing[0];
            const real yj = X1[1] + ((real) j - 0.5) * g.spacing[1];
            const real e = std::exp(-d * nu * t);
            if (three_d) {
                const real zk = X1[2] + ((real) k - 0.5) * g.spacing[2];
                const real s = std::sin(xi + yj + zk);
                u[(size_t) idx] = e * s;
                v[(size_t) idx] = -0.5 * e * s;
                w[(size_t) idx] = -0.5 * e * s;
            } else {
                const real s = std::sin(xi + yj);
                u[(size_t) idx] = e * s;
                v[(size_t) idx] = -e * s;
                w[(size_t) idx] = 0.;
            }
        }
        m_fc->u.from_host(u);
        m_fc->v.from_host(v);
        m_fc->w.from_host(w);
    } else if (ic.usr_fct == "SinSinSin") {
        // Functions::sin_sin_sin (src/Functions.cpp:782-812)
        m_fc->p.set_value(0.);
        const GridLevel &g = geo.grid().level(0);
        const auto &X1 = geo.grid().start_pd;
        std::vector<real> rhs = m_fc->rhs.to_host();
        const size_t Nx = g.N[0], Nxy = g.N[0] * g.N[1];
        const double l = ic.sin_l;
        for (Idx idx : inner) {
            const size_t k = (size_t) idx / Nxy, j = ((size_t) idx - k * Nxy) / Nx, i = (size_t) idx - k * Nxy - j * Nx;
            const double xi = X1[0] + ((double) i - 0.5) * g.spacing[0];
            const double yj = X1[1] + ((double) j - 0.5) * g.spacing[1];
            const double zk = X1[2] + ((double) k - 0.5) * g.spacing[2];
            rhs[(size_t) idx] = std::sin(l * M_PI * xi) * std::sin(l * M_PI * yj) * std::sin(l * M_PI * zk);
        }
        m_fc->rhs.from_host(rhs);
    } else if (ic.usr_fct == "ExpSinusProd" || ic.usr_fct == "GaussBubble" || ic.usr_fct == "Hat") {
        // Functions::exp_sinus_prod / gauss_bubble / hat (src/Functions.cpp:324-353,
        // 471-511, hat) at t = 0 on the inner cells of u, v and w
        const GridLevel &g = geo.grid().level(0);
        const auto &X1 = geo.grid().start_pd;
        const size_t Nx = g.N[0], Nxy = g.N[0] * g.N[1];
        auto num = [&](const char *k) { return std::stod(ic.values.at(k)); };
        const real t = 0.;
        std::vector<real> out(m_fc->u.get_size());
        for (Idx idx : inner) {
            const size_t k = (size_t) idx / Nxy, j = ((size_t) idx - k * Nxy) / Nx, i = (size_t) idx - k * Nxy - j * Nx;
            const real xi = X1[0] + ((real) i - 0.5) * g.spacing[0];
            const real yj = X1[1] + ((real) j - 0.5) * g.spacing[1];
            const real zk = X1[2] + ((real) k - 0.5) * g.spacing[2];
            real v;
            if (ic.usr_fct == "ExpSinusProd") {
                const real A = 1.0, l = num("l");
                const real kpinu = 3 * l * l * M_PI * M_PI * m_rt.settings().physical.nu.value_or(0.0);
                v = A * std::exp(-kpinu * t) * std::sin(l * M_PI * xi) * std::sin(l * M_PI * yj) *
                    std::sin(l * M_PI * zk);
            } else if (ic.usr_fct == "GaussBubble") {
                const real u_lin = num("u_lin"), v_lin = num("v_lin"), w_lin = num("w_lin");
                const real l = num("l");
                const real xs = (xi - num("x_shift")) / u_lin - t, ys = (yj - num("y_shift")) / v_lin - t;
                const real x2 = xs * xs, y2 = ys * ys;
                real z2 = 0;
                if (w_lin != 0) {
                    const real zs = (zk - num("z_shift")) / w_lin - t;
                    z2 = zs * zs;
                }
                const real quot = 1. / (2. * l * l);
                v = std::exp(-(x2 + y2 + z2) * quot);
            } else {
                const bool in = (num("x1") <= xi && xi <= num("x2")) && (num("y1") <= yj && yj <= num("y2")) &&
                                (num("z1") <= zk && zk <= num("z2"));
                v = in ? num("val_in") : num("val_out");
            }
            out[(size_t) idx] = v;
        }
        for (Field *f : {&m_fc->u, &m_fc->v, &m_fc->w}) {
            std::vector<real> h = f->to_host();
            for (Idx idx : inner) h[(size_t) idx] = out[(size_t) idx];
            f->from_host(h);
        }
    } else if (ic.usr_fct == "Drift" || ic.usr_fct == "McDermott" || ic.usr_fct == "Vortex") {
        // the Navier-Stokes test states on the inner cells of u, v, w and p:
        // Functions::drift (src/Functions.cpp:297-317), Functions::mcdermott
        // (:696-729, at t = 0) and Functions::vortex (:842-886); McDermott and
        // Vortex are followed by p = 0 everywhere (SolverController.cpp:130-148)
        const GridLevel &g = geo.grid().level(0);
        const auto &X1 = geo.grid().start_pd;
        const size_t Nx = g.N[0], Nxy = g.N[0] * g.N[1];
        auto num = [&](const char *k) { return std::stod(ic.values.at(k)); };
        std::vector<real> u = m_fc->u.to_host(), v = m_fc->v.to_host(), w = m_fc->w.to_host(), p = m_fc->p.to_host();
        auto xi = [&](size_t i) { return X1[0] + ((real) i - 0.5) * g.spacing[0]; };
        auto yj = [&](size_t j) { return X1[1] + ((real) j - 0.5) * g.spacing[1]; };
        if (ic.usr_fct == "Drift") {
            const real u_lin = num("u_lin"), v_lin = num("v_lin"), w_lin = num("w_lin"), pa = num("pa");
            for (Idx idx : inner) {
                u[(size_t) idx] = u_lin;
                v[(size_t) idx] = v_lin;
                w[(size_t) idx] = w_lin;
                p[(size_t) idx] = pa;
            }
        } else if (ic.usr_fct == "McDermott") {
            const real A = num("A"), nu = m_rt.settings().physical.nu.value(), t = 0.;
            for (Idx idx : inner) {
                const size_t k = (size_t) idx / Nxy, j = ((size_t) idx - k * Nxy) / Nx, i = (size_t) idx - k * Nxy - j * Nx;
                u[(size_t) idx] = 1. - A * std::cos(xi(i) - t) * std::sin(yj(j) - t) * std::exp(-2 * nu * t);
                v[(size_t) idx] = 1. + A * std::sin(xi(i) - t) * std::cos(yj(j) - t) * std::exp(-2 * nu * t);
                w[(size_t) idx] = 0.;
                p[(size_t) idx] = -0.25 * A * A * (std::cos(2 * (xi(i) - t)) + std::cos(2 * (yj(j) - t))) *
                                  std::exp(-4 * nu * t);
            }
        } else {
            // the reference reads the vortex's v from w_lin and its w from v_lin
            const real u_lin = num("u_lin"), v_lin = num("w_lin"), rhoa = num("rhoa"), pa = num("pa");
            const real L = geo.grid().length_cd(0);
            const real R_c = L / 20.;
            const real G = 0.04 * u_lin * R_c * std::sqrt(std::exp(1));
            const real GrR_c = G / (R_c * R_c);
            const real rR_c = 1. / (2. * R_c * R_c);
            const real rhoGrR_c = rhoa * G * G * rR_c;
            for (Idx idx : inner) {
                const size_t k = (size_t) idx / Nxy, j = ((size_t) idx - k * Nxy) / Nx, i = (size_t) idx - k * Nxy - j * Nx;
                const real x = xi(i), y = yj(j);
                u[(size_t) idx] = u_lin - GrR_c * y * std::exp(-rR_c * (x * x + y * y));
                v[(size_t) idx] = v_lin + GrR_c * x * std::exp(-rR_c * (x * x + y * y));
                w[(size_t) idx] = 0.;
                p[(size_t) idx] = pa - rhoGrR_c * std::exp(-rR_c * (x * x + y * y));
            }
        }
        m_fc->u.from_host(u);
        m_fc->v.from_host(v);
        m_fc->w.from_host(w);
        m_fc->p.from_host(p);
        if (ic.usr_fct != "Drift") m_fc->p.set_value(0.);
    } else if (ic.usr_fct != "Zero") {
        // Jet (Functions::jet, src/Functions.cpp:658-688) measures its end indices from the
        // END of the physical domain, so every end coordinate inside the domain gives a
        // negative index converted to size_t, and its axis loops run to number_of_axes
        // inclusive; no reference configuration uses it
        throw config_error("initial condition '" + ic.usr_fct +
                           "' is not one of Uniform, LayersT, SinSinSin, ExpSinusProd, ExpSinusSum, GaussBubble, Hat, "
                           "Drift, McDermott, Vortex, Zero (the initial conditions of the solvers this library runs)");
    }
    const std::string &d = m_rt.settings().solver.description;
    if (d == "NSTempTurbSolver" || d == "NSTempSolver" || d == "NSTempTurbConSolver" || d == "NSTempConSolver")
        force_source();
}

void SolverController::force_source() {
    // SolverController::force_source (src/solver/SolverController.cpp:229-257)
    const auto &src = m_rt.settings().solver.source;
    if (src.force_fct == "Buoyancy") {
        if (!src.use_init_values) m_fc->T_ambient.set_value(src.ambient_temperature.value());
    } else if (src.force_fct == "Uniform") {
        // Functions::uniform on the force components named by dir, inner cells only
        const IdxList &inner = m_rt.geometry().inner(0);
        Field *force[3] = {&m_fc->f_x, &m_fc->f_y, &m_fc->f_z};
        for (int a = 0; a < 3; a++) {
            if (std::find(src.dir.begin(), src.dir.end(), a) == src.dir.end()) continue;
            std::vector<real> h = force[a]->to_host();
            for (Idx idx : inner) h[(size_t) idx] = src.uniform_value[a];
            force[a]->from_host(h);
        }
    }
}

void SolverController::momentum_source() {
    // SolverController::momentum_source (src/solver/SolverController.cpp:263-284)
    const auto &dir = m_rt.settings().solver.source.dir;
    auto has = [&](int a) { return std::find(dir.begin(), dir.end(), a) != dir.end(); };
    if (has(AXIS_X)) ISource::buoyancy_force(m_fc->f_x, m_fc->T, m_fc->T_ambient);
    if (has(AXIS_Y)) ISource::buoyancy_force(m_fc->f_y, m_fc->T, m_fc->T_ambient);
    if (has(AXIS_Z)) ISource::buoyancy_force(m_fc->f_z, m_fc->T, m_fc->T_ambient);
}

void SolverController::update_sources(real t_cur, bool) {
    if (m_has_momentum_source && m_rt.settings().solver.source.force_fct == "Buoyancy") momentum_source();
    m_solver->update_source(t_cur);
}

// ---------------------------------------------------------------- TimeIntegration

TimeIntegration::TimeIntegration(Runtime &rt, SolverController &sc)
    : m_rt(rt), m_sc(sc), m_dt(rt.settings().physical.dt), m_t_end(rt.settings().physical.t_end), m_t_cur(m_dt) {}

bool TimeIntegration::finished() const { return !(m_t_cur < m_t_end + m_dt / 2); }

void TimeIntegration::set_step(int64_t step) {
    if (step < 1) throw std::invalid_argument("step index starts at 1");
    m_step = step;
    m_t_cur = (real) m_step * m_dt;  // as run() advances it
}

void TimeIntegration::step_io(const std::vector<std::pair<Field *, const real *>> &in,
                              const std::vector<std::pair<Field *, real *>> &out) {
    if (finished()) throw std::logic_error("the simulation has reached t_end");
    StepIO io(m_rt.ctx());
    // NSTempTurbSolver / NSTempSolver read p and T late: those arrive on the
    // second stream during the step; the rest before it
    const bool late_ok = dynamic_cast<NSTempTurbSolver *>(&m_sc.solver()) != nullptr;
    FieldController &fc = m_sc.fields();
    bool vel = false, temp_now = false;
    for (const auto &i : in) {
        if (late_ok && (i.first == &fc.p || i.first == &fc.T)) continue;
        check(artss_upload_async(m_rt.ctx(), i.first->data, i.second, (int64_t) i.first->get_size()), "upload");
        vel = vel || i.first == &fc.u || i.first == &fc.v || i.first == &fc.w;
        temp_now = temp_now || i.first == &fc.T;
    }
    // uploaded u, v, w (T) are the state the step advances: their copies
    // follow, as FieldController::update_data sets them after a step
    if (vel) FieldController::couple_vector(fc.u, fc.u0, fc.u_tmp, fc.v, fc.v0, fc.v_tmp, fc.w, fc.w0, fc.w_tmp);
    if (temp_now) FieldController::couple_scalar(fc.T, fc.T0, fc.T_tmp);
    for (const auto &i : in)
        if (late_ok && (i.first == &fc.p || i.first == &fc.T)) io.upload_late(*i.first, i.second);
    for (const auto &o : out) io.add_output(*o.first, o.second);
    m_rt.io = &io;
    try {
        run(1);
    } catch (...) {
        m_rt.io = nullptr;
        throw;
    }
    m_rt.io = nullptr;
    io.finish();
}

void TimeIntegration::step_io_async(const std::vector<std::pair<Field *, const real *>> &in,
                                    const std::vector<std::pair<Field *, real *>> &out) {
    if (finished()) throw std::logic_error("the simulation has reached t_end");
    artss_ctx *ctx = m_rt.ctx();
    FieldController &fc = m_sc.fields();
    const int64_t n = (int64_t) fc.u.get_size();
    std::vector<double *> in_dev;
    std::vector<const double *> in_host;
    bool vel = false, temp = false;
    for (const auto &i : in) {
        if ((int64_t) i.first->get_size() != n) throw std::invalid_argument("step_io_async: level-0 fields only");
        in_dev.push_back(i.first->data);
        in_host.push_back(i.second);
        vel = vel || i.first == &fc.u || i.first == &fc.v || i.first == &fc.w;
        temp = temp || i.first == &fc.T;
    }
    check(artss_io_in(ctx, (int) in.size(), in_dev.data(), in_host.data(), n), "io_in");
    // uploaded u, v, w, T are the state the step advances (as in step_io); p
    // and T set at the start instead of during the velocity: nothing of the
    // step reads them before (the buoyancy force was formed from the previous T)
    if (vel) FieldController::couple_vector(fc.u, fc.u0, fc.u_tmp, fc.v, fc.v0, fc.v_tmp, fc.w, fc.w0, fc.w_tmp);
    if (temp) FieldController::couple_scalar(fc.T, fc.T0, fc.T_tmp);
    run(1);
    std::vector<const double *> out_dev;
    std::vector<double *> out_host;
    for (const auto &o : out) {
        if ((int64_t) o.first->get_size() != n) throw std::invalid_argument("step_io_async: level-0 fields only");
        out_dev.push_back(o.first->data);
        out_host.push_back(o.second);
    }
    check(artss_io_out(ctx, (int) out.size(), out_dev.data(), out_host.data(), n), "io_out");
}

TimeIntegration::~TimeIntegration() { artss_graph_destroy(m_graph); }

void TimeIntegration::capture_step() {
    artss_ctx *ctx = m_rt.ctx();
    if (artss_graph_begin(ctx) != ARTSS_OK) {
        m_graph_failed = true;
        return;
    }
    bool ok = true;
    try {
        m_sc.solver_do_step(m_t_cur, false);
        m_sc.update_sources(m_t_cur, false);
        m_sc.fields().update_data();
    } catch (const std::exception &) {
        ok = false;
    }
    if (!ok || artss_graph_end(ctx, 0, &m_graph) != ARTSS_OK) {
        if (!ok) artss_graph_end(ctx, 1, nullptr);
        m_graph = nullptr;
        m_graph_failed = true;
    }
}

int64_t TimeIntegration::run(int64_t steps) {
    int64_t done = 0;
    while (!finished() && (steps < 0 || done < steps)) {
        if (m_rt.graphs && m_step >= kGraphStep && !m_graph_failed && !m_rt.io) {
            if (!m_graph) capture_step();
            if (m_graph) {
                for (auto &p : m_rt.step_params) p(m_t_cur);
                check(artss_graph_launch(m_graph), "step graph");
                graph_steps++;
                m_step++;
                m_t_cur = (real) m_step * m_dt;
                done++;
                continue;
            }
        }
        m_sc.solver_do_step(m_t_cur, false);
        artss_ctx_stage_mark(m_rt.ctx(), ARTSS_STAGE_UPDATE);
        m_sc.update_sources(m_t_cur, false);
        m_sc.fields().update_data();
        artss_ctx_stage_mark(m_rt.ctx(), ARTSS_STAGE_END);
        m_step++;
        m_t_cur = (real) m_step * m_dt;
        done++;
    }
    return done;
}

}  // namespace artss
