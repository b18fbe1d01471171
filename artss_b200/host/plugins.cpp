#include "plugins.h"

#include <cmath>

namespace artss {

// ---------------------------------------------------------------- IPressure

void IPressure::divergence(Field &out, const Field &in_x, const Field &in_y, const Field &in_z, bool) {
    check(artss_divergence(out.runtime().ctx(), out.data, in_x.data, in_y.data, in_z.data), "divergence");
}

void IPressure::projection(Field &out_u, Field &out_v, Field &out_w, const Field &in_u, const Field &in_v,
                           const Field &in_w, const Field &in_p, bool) {
    check(artss_projection(out_u.runtime().ctx(), out_u.data, out_v.data, out_w.data, in_u.data, in_v.data,
                           in_w.data, in_p.data),
          "projection");
}

// ---------------------------------------------------------------- ISource

void ISource::buoyancy_force(Field &out, const Field &in, const Field &in_a, bool) {
    const auto &phys = out.runtime().settings().physical;
    check(artss_buoyancy_force(out.runtime().ctx(), out.data, in.data, in_a.data, phys.beta, phys.g),
          "buoyancy_force");
}

// ---------------------------------------------------------------- SLAdvect

void SLAdvect::advect(Field &out, const Field &in, const Field &u_vel, const Field &v_vel, const Field &w_vel, bool) {
    check(artss_advect_sl(m_rt.ctx(), out.data, in.data, u_vel.data, v_vel.data, w_vel.data, m_rt.dt(),
                          out.get_type()),
          "SLAdvect::advect");
}

void SLAdvect::advect_vector(Field &out_u, Field &out_v, Field &out_w, const Field &in_u, const Field &in_v,
                             const Field &in_w, const Field &u_vel, const Field &v_vel, const Field &w_vel) {
    check(artss_advect_sl_uvw(m_rt.ctx(), out_u.data, out_v.data, out_w.data, in_u.data, in_v.data, in_w.data,
                              u_vel.data, v_vel.data, w_vel.data, m_rt.dt()),
          "SLAdvect::advect_vector");
}

// ---------------------------------------------------------------- diffusion

void ColoredGaussSeidelDiffuse::run(Field &out, const Field &in, const Field &b, real D, const Field *ev) {
    artss_iter_cfg cfg{(int64_t) m_settings.max_iter, m_settings.tol_res, m_settings.w};
    artss_iter_stats st{};
    // the reference overwrites its const `in` argument (ColoredGaussSeidelDiffuse.cpp:71)
    const int flags = (in_is_scratch ? ARTSS_DIFFUSE_IN_SCRATCH : 0) | (out_holds_in ? ARTSS_DIFFUSE_OUT_HOLDS_IN : 0);
    if (m_mixed)
        check(artss_diffuse_cgs_mixed(m_rt.ctx(), out.data, in.data, b.data, D, ev ? ev->data : nullptr, m_rt.dt(),
                                      out.get_type(), &cfg, flags, &st),
              "ColoredGaussSeidelDiffuse::diffuse (mixed precision)");
    else
        check(artss_diffuse_cgs(m_rt.ctx(), out.data, in.data, b.data, D, ev ? ev->data : nullptr, m_rt.dt(),
                                out.get_type(), &cfg, flags, &st),
              "ColoredGaussSeidelDiffuse::diffuse");
    last_iterations = st.iterations;
    last_residual = st.residual;
}

void ColoredGaussSeidelDiffuse::diffuse(Field &out, const Field &in, const Field &b, real D, bool) {
    run(out, in, b, D, nullptr);
}

void ColoredGaussSeidelDiffuse::diffuse(Field &out, const Field &in, const Field &b, real D, const Field &ev, bool) {
    run(out, in, b, D, &ev);
}

void ExplicitDiffuse::diffuse(Field &out, const Field &in, const Field &, real D, bool) {
    check(artss_diffuse_explicit(m_rt.ctx(), out.data, in.data, D, nullptr, m_rt.dt(), out.get_type()),
          "ExplicitDiffuse::diffuse");
    last_iterations = 1;
}

void ExplicitDiffuse::diffuse(Field &out, const Field &in, const Field &, real D, const Field &ev, bool) {
    check(artss_diffuse_explicit(m_rt.ctx(), out.data, in.data, D, ev.data, m_rt.dt(), out.get_type()),
          "ExplicitDiffuse::diffuse");
    last_iterations = 1;
}

void JacobiDiffuse::run(Field &out, const Field &in, const Field &b, real D, const Field *ev) {
    artss_iter_cfg cfg{(int64_t) m_settings.max_iter, m_settings.tol_res, m_settings.w};
    artss_iter_stats st{};
    check(artss_diffuse_jacobi(m_rt.ctx(), out.data, in.data, b.data, D, ev ? ev->data : nullptr, m_rt.dt(),
                               out.get_type(), &cfg, &st),
          "JacobiDiffuse::diffuse");
    last_iterations = st.iterations;
    last_residual = st.residual;
}

void JacobiDiffuse::diffuse(Field &out, const Field &in, const Field &b, real D, bool) { run(out, in, b, D, nullptr); }

void JacobiDiffuse::diffuse(Field &out, const Field &in, const Field &b, real D, const Field &ev, bool) {
    run(out, in, b, D, &ev);
}

// ---------------------------------------------------------------- VCycleMG

VCycleMG::VCycleMG(Runtime &rt, const settings::Pressure &s, bool to_rel_tol)
    : m_rt(rt), m_settings(s), m_rel(to_rel_tol) {
    artss_mg_cfg c{};
    c.n_level = (int32_t) s.n_level;
    c.n_cycle = (int32_t) s.n_cycle;
    c.max_cycle = (int32_t) s.max_cycle;
    c.n_relax = (int32_t) s.n_relax;
    c.tol_res = s.tol_res;
    if (s.smoother.type == "Jacobi") c.smoother = ARTSS_SMOOTHER_JACOBI;
    else if (s.smoother.type == "ColoredGaussSeidel") c.smoother = ARTSS_SMOOTHER_CGS;
    else throw config_error("VCycleMG smoother '" + s.smoother.type + "' is not implemented");
    c.smoother_max_iter = (int64_t) s.smoother.max_iter;
    c.smoother_tol_res = s.smoother.tol_res;
    c.smoother_w = s.smoother.w;
    check(artss_mg_create(rt.ctx(), &c, &m_mg), "VCycleMG");
}

VCycleMG::~VCycleMG() { artss_mg_destroy(m_mg); }

void VCycleMG::pressure(Field &out, const Field &b, real t, bool) {
    if (m_rel) {
        artss_solve_stats st{};
        check(artss_mg_solve_rel(m_mg, out.data, b.data, m_settings.tol_res, (int64_t) m_settings.max_cycle, &st),
              "VCycleMGRel::pressure");
        last_cycles = st.cycles;
        last_residual = st.residual;
        return;
    }
    // VCycleMG::pressure (src/pressure/VCycleMG.cpp:142-207): Nt == 1 iterates to tolerance
    const auto Nt = static_cast<size_t>(std::round(t / m_rt.dt()));
    artss_mg_stats st{};
    check(artss_mg_pressure(m_mg, out.data, b.data, Nt == 1 ? 1 : 0, &st), "VCycleMG::pressure");
    last_cycles = st.cycles;
    last_residual = st.residual;
}

// ---------------------------------------------------------------- VCycleMGMixed

MixedVCycle::MixedVCycle(Runtime &rt, const settings::Pressure &s) : m_rt(rt) {
    artss_mixed_cfg c{};
    c.n_level = (int32_t) s.n_level;
    c.n_relax = (int32_t) s.n_relax;
    c.coarse_smoother = ARTSS_SMOOTHER_CGS;
    c.flags = 0;
    c.w = s.smoother.w;
    c.coarse_w = 0.0;  // red-black SOR, optimal weight of the model problem
    c.coarse_rel_tol = 1e-3;
    c.coarse_max_iter = 40;
    c.rel_tol = s.tol_res;
    c.max_cycles = (int64_t) s.max_cycle;
    check(artss_mixed_create(rt.ctx(), &c, &m_mx), "VCycleMGMixed");
}

MixedVCycle::~MixedVCycle() { artss_mixed_destroy(m_mx); }

void MixedVCycle::pressure(Field &out, const Field &b, real, bool) {
    artss_solve_stats st{};
    check(artss_mixed_solve(m_mx, out.data, b.data, &st), "VCycleMGMixed::pressure");
    last_cycles = st.cycles;
    last_residual = st.residual;
}

// ---------------------------------------------------------------- turbulence / sources

void ConstSmagorinsky::calc_turbulent_viscosity(Field &ev, const Field &in_u, const Field &in_v, const Field &in_w,
                                                bool) {
    check(artss_turb_const_smagorinsky(m_rt.ctx(), ev.data, in_u.data, in_v.data, in_w.data, m_cs),
          "ConstSmagorinsky");
}

void DynamicSmagorinsky::calc_turbulent_viscosity(Field &ev, const Field &in_u, const Field &in_v, const Field &in_w,
                                                  bool) {
    check(artss_turb_dynamic_smagorinsky(m_rt.ctx(), ev.data, in_u.data, in_v.data, in_w.data,
                                         m_rt.settings().physical.nu.value()),
          "DynamicSmagorinsky");
}

void ExplicitEulerSource::add_source(Field &out_x, Field &out_y, Field &out_z, const Field &S_x, const Field &S_y,
                                     const Field &S_z, bool) {
    // ExplicitEulerSource.cpp:40-96: only the axes listed in `dir`, in x, y, z order
    Field *outs[3] = {&out_x, &out_y, &out_z};
    const Field *srcs[3] = {&S_x, &S_y, &S_z};
    for (int a = 0; a < 3; a++) {
        bool on = false;
        for (int d : m_dir) on = on || d == a;
        if (!on) continue;
        check(artss_add_source(m_rt.ctx(), outs[a]->data, srcs[a]->data, m_rt.dt(), outs[a]->get_type()),
              "ExplicitEulerSource::add_source");
    }
}

void ExplicitEulerSource::dissipate(Field &out, const Field &in_u, const Field &in_v, const Field &in_w, bool) {
    const auto &phys = m_rt.settings().physical;
    check(artss_dissipate(m_rt.ctx(), out.data, in_u.data, in_v.data, in_w.data, phys.nu.value(), m_rt.dt(),
                          out.get_type()),
          "ISource::dissipate");
}

void ExplicitEulerSource::add_source(Field &out, const Field &S, bool) {
    check(artss_add_source(m_rt.ctx(), out.data, S.data, m_rt.dt(), out.get_type()), "ExplicitEulerSource::add_source");
}

// ---------------------------------------------------------------- Gauss source

GaussFunction::GaussFunction(Runtime &rt, const settings::Gauss &s) : m_rt(rt), m_settings(s), m_spatial(rt, F_RHO) {
    create_spatial_values();
}

void GaussFunction::create_spatial_values() {
    // GaussFunction::create_spatial_values (src/source/GaussFunction.cpp:53-107), on the host
    const Geometry &geo = m_rt.geometry();
    const GridLevel &g = geo.grid().level(0);
    const auto &X1 = geo.grid().start_pd;
    std::array<double, 3> r_sigma{};
    for (int a = 0; a < 3; a++) {
        r_sigma[a] = m_settings.dimension[a] * m_settings.dimension[a];
        r_sigma[a] *= 2;
        r_sigma[a] = 1. / r_sigma[a];
    }
    std::array<size_t, 3> src{};
    for (int a = 0; a < 3; a++)
        src[a] = (size_t) (std::round((-X1[a] + m_settings.position[a]) / g.spacing[a]) + 1);
    const IdxList &inner = geo.inner(0);
    const size_t Nx = g.N[0], Nxy = g.N[0] * g.N[1];
    auto expr_at = [&](Idx idx, bool &blocked) {
        const size_t k = (size_t) idx / Nxy;
        const size_t j = ((size_t) idx - k * Nxy) / Nx;
        const size_t i = (size_t) idx - k * Nxy - j * Nx;
        const std::array<size_t, 3> c{i, j, k};
        blocked = geo.blocked(src, c);
        double delta[3];
        for (int a = 0; a < 3; a++) {
            const double mid = X1[a] + ((double) c[a] - 0.5) * g.spacing[a];
            delta[a] = mid - m_settings.position[a];
            delta[a] *= delta[a];
            delta[a] *= r_sigma[a];
        }
        return std::exp(-(delta[0] + delta[1] + delta[2]));
    };
    double V = 0.;
    for (Idx idx : inner) {
        bool blocked;
        const double e = expr_at(idx, blocked);
        if (blocked) continue;
        V += e * g.spacing[0] * g.spacing[1] * g.spacing[2];
    }
    const double HRRrV = m_settings.heat_release_rate / V;
    const double rcp = 1. / m_settings.heat_capacity;
    std::vector<double> values(m_spatial.get_size(), 0.0);
    for (Idx idx : inner) {
        bool blocked;
        const double e = expr_at(idx, blocked);
        if (blocked) continue;
        values[(size_t) idx] = HRRrV * rcp * e;
    }
    m_spatial.from_host(values);
}

void GaussFunction::update_source(Field &out, real t_cur) {
    // GaussFunction::update_source (src/source/GaussFunction.cpp:27-40)
    if (m_rt.capturing()) {
        // a captured step: the factor comes from a parameter slot set before each replay
        if (m_noise) throw std::runtime_error("a source with noise cannot be captured");
        if (m_param < 0) {
            m_param = m_rt.next_param_slot++;
            const real tau = m_settings.tau;
            artss_ctx *ctx = m_rt.ctx();
            const int slot = m_param;
            m_rt.step_params.push_back(
                [ctx, slot, tau](real t) { check(artss_param_set(ctx, slot, std::tanh(t / tau)), "source factor"); });
        }
        check(artss_scale_copy_param(m_rt.ctx(), out.data, m_spatial.data, m_param, 0), "source");
        return;
    }
    const real time_val = std::tanh(t_cur / m_settings.tau);
    // out.copy_data(spatial); out *= time_val; as one pass (the same product)
    check(artss_scale_copy(m_rt.ctx(), out.data, m_spatial.data, time_val, (int) out.get_level()), "source");
    if (m_noise) {
        std::vector<real> noise = m_noise->random_field(out.get_size());
        if (m_absolute) {
            std::vector<real> cur = out.to_host();
            for (size_t i = 0; i < cur.size(); i++) cur[i] += noise[i];
            out.from_host(cur);
        } else {
            std::vector<real> cur = out.to_host();
            for (size_t i = 0; i < cur.size(); i++) cur[i] *= (noise[i] + 1);
            out.from_host(cur);
        }
    }
}

void GaussFunction::update_obstacle_change() {
    m_spatial.set_value(0);
    create_spatial_values();
}

}  // namespace artss
