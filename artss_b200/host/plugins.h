// The ARTSS plugin interfaces (ARTSS src/interfaces/*.h) with their method
// signatures unchanged, and the implementations of the fractional-step path,
// each a thin adapter over one C-ABI entry point of include/artss_cuda.h.
#pragma once

#include <memory>
#include <random>
#include <string>
#include <vector>

#include "runtime.h"

namespace artss {

// IAdvection (src/interfaces/IAdvection.h:12-17)
class IAdvection {
 public:
    virtual ~IAdvection() = default;
    virtual void advect(Field &out, const Field &in, const Field &u_vel, const Field &v_vel, const Field &w_vel,
                        bool sync) = 0;
};

// IDiffusion (src/interfaces/IDiffusion.h:13-20)
class IDiffusion {
 public:
    virtual ~IDiffusion() = default;
    virtual void diffuse(Field &out, const Field &in, const Field &b, real D, bool sync) = 0;
    virtual void diffuse(Field &out, const Field &in, const Field &b, real D, const Field &ev, bool sync) = 0;
    // iterations and final residual of the last call
    int64_t last_iterations = 0;
    double last_residual = 0;
    // Declares that `in` is dead after diffuse() (the caller overwrites it
    // before reading), letting the solver skip the per-sweep snapshot copy.
    bool in_is_scratch = false;
    bool out_holds_in = false;  // the caller coupled out and in from one field before diffuse()
};

// IPressure (src/interfaces/IPressure.h:13-25)
class IPressure {
 public:
    virtual ~IPressure() = default;
    virtual void pressure(Field &out, const Field &b, real t, bool sync) = 0;
    void divergence(Field &out, const Field &in_x, const Field &in_y, const Field &in_z, bool sync);
    void projection(Field &out_u, Field &out_v, Field &out_w, const Field &in_u, const Field &in_v,
                    const Field &in_w, const Field &in_p, bool sync);
    int64_t last_cycles = 0;
    double last_residual = -1;
};

// ITurbulence (src/interfaces/ITurbulence.h:12-23)
class ITurbulence {
 public:
    virtual ~ITurbulence() = default;
    virtual void calc_turbulent_viscosity(Field &ev, const Field &in_u, const Field &in_v, const Field &in_w,
                                          bool sync) = 0;
    virtual void explicit_filtering(Field &out, const Field &in, bool sync) = 0;
};

// ISource (src/interfaces/ISource.h:14-30)
class ISource {
 public:
    virtual ~ISource() = default;
    virtual void add_source(Field &out_x, Field &out_y, Field &out_z, const Field &S_x, const Field &S_y,
                            const Field &S_z, bool sync) = 0;
    virtual void add_source(Field &out, const Field &S, bool sync) = 0;
    static void buoyancy_force(Field &out, const Field &in, const Field &in_a, bool sync = true);
    // viscous dissipation into out (ISource::dissipate, src/interfaces/ISource.cpp:63-123)
    virtual void dissipate(Field &out, const Field &in_u, const Field &in_v, const Field &in_w, bool sync) = 0;
};

// ISourceFunction (src/interfaces/ISourceFunction.h:14-29)
class ISourceFunction {
 public:
    virtual ~ISourceFunction() = default;
    virtual void update_source(Field &out, real t_cur) = 0;
    virtual void update_obstacle_change() = 0;
};

// ---------------------------------------------------------------- implementations

class SLAdvect : public IAdvection {
 public:
    explicit SLAdvect(Runtime &rt) : m_rt(rt) {}
    void advect(Field &out, const Field &in, const Field &u_vel, const Field &v_vel, const Field &w_vel,
                bool sync) override;
    // three advect() calls sharing one backtrace (u,v,w advected by the same velocity)
    void advect_vector(Field &out_u, Field &out_v, Field &out_w, const Field &in_u, const Field &in_v,
                       const Field &in_w, const Field &u_vel, const Field &v_vel, const Field &w_vel);

 private:
    Runtime &m_rt;
};

class ColoredGaussSeidelDiffuse : public IDiffusion {
 public:
    // mixed: FP32 sweeps inside FP64 defect correction (artss_diffuse_cgs_mixed),
    // the XML type ColoredGaussSeidelMixed (same keys)
    ColoredGaussSeidelDiffuse(Runtime &rt, const settings::Diffusion &s, bool mixed = false)
        : m_rt(rt), m_settings(s), m_mixed(mixed) {}
    void diffuse(Field &out, const Field &in, const Field &b, real D, bool sync) override;
    void diffuse(Field &out, const Field &in, const Field &b, real D, const Field &ev, bool sync) override;

 private:
    void run(Field &out, const Field &in, const Field &b, real D, const Field *ev);
    Runtime &m_rt;
    settings::Diffusion m_settings;
    bool m_mixed;
};

// ExplicitDiffuse (src/diffusion/ExplicitDiffuse.cpp:27-127): one explicit step per call
class ExplicitDiffuse : public IDiffusion {
 public:
    explicit ExplicitDiffuse(Runtime &rt) : m_rt(rt) {}
    void diffuse(Field &out, const Field &in, const Field &b, real D, bool sync) override;
    void diffuse(Field &out, const Field &in, const Field &b, real D, const Field &ev, bool sync) override;

 private:
    Runtime &m_rt;
};

class JacobiDiffuse : public IDiffusion {
 public:
    JacobiDiffuse(Runtime &rt, const settings::Diffusion &s) : m_rt(rt), m_settings(s) {}
    void diffuse(Field &out, const Field &in, const Field &b, real D, bool sync) override;
    void diffuse(Field &out, const Field &in, const Field &b, real D, const Field &ev, bool sync) override;

 private:
    void run(Field &out, const Field &in, const Field &b, real D, const Field *ev);
    Runtime &m_rt;
    settings::Diffusion m_settings;
};

class VCycleMG : public IPressure {
 public:
    // to_rel_tol: every call repeats the reference V-cycle until the relative
    // residual ||b - A p|| / ||b|| <= tol_res (at most max_cycle cycles): the XML
    // type VCycleMGRel, the FP64 counterpart of VCycleMGMixed
    VCycleMG(Runtime &rt, const settings::Pressure &s, bool to_rel_tol = false);
    ~VCycleMG() override;
    void pressure(Field &out, const Field &b, real t, bool sync) override;
    artss_mg *handle() const { return m_mg; }

 private:
    Runtime &m_rt;
    settings::Pressure m_settings;
    artss_mg *m_mg = nullptr;
    bool m_rel = false;
};

// Mixed-precision pressure solve (no reference counterpart; artss_mixed_*):
// every call iterates FP32 V-cycles inside FP64 defect correction from the
// current pressure until ||b - A p|| <= tol_res ||b|| or max_cycle cycles.
class MixedVCycle : public IPressure {
 public:
    MixedVCycle(Runtime &rt, const settings::Pressure &s);
    ~MixedVCycle() override;
    void pressure(Field &out, const Field &b, real t, bool sync) override;

 private:
    Runtime &m_rt;
    artss_mixed *m_mx = nullptr;
};

class ConstSmagorinsky : public ITurbulence {
 public:
    ConstSmagorinsky(Runtime &rt, real cs) : m_rt(rt), m_cs(cs) {}
    void calc_turbulent_viscosity(Field &ev, const Field &in_u, const Field &in_v, const Field &in_w,
                                  bool sync) override;
    void explicit_filtering(Field &, const Field &, bool) override {}

 private:
    Runtime &m_rt;
    real m_cs;
};

// DynamicSmagorinsky (src/turbulence/DynamicSmagorinsky.cpp:172-427); nu from the settings
class DynamicSmagorinsky : public ITurbulence {
 public:
    explicit DynamicSmagorinsky(Runtime &rt) : m_rt(rt) {}
    void calc_turbulent_viscosity(Field &ev, const Field &in_u, const Field &in_v, const Field &in_w,
                                  bool sync) override;
    void explicit_filtering(Field &, const Field &, bool) override {}

 private:
    Runtime &m_rt;
};

class ExplicitEulerSource : public ISource {
 public:
    ExplicitEulerSource(Runtime &rt, std::vector<int> dir) : m_rt(rt), m_dir(std::move(dir)) {}
    void add_source(Field &out_x, Field &out_y, Field &out_z, const Field &S_x, const Field &S_y, const Field &S_z,
                    bool sync) override;
    void add_source(Field &out, const Field &S, bool sync) override;
    void dissipate(Field &out, const Field &in_u, const Field &in_v, const Field &in_w, bool sync) override;

 private:
    Runtime &m_rt;
    std::vector<int> m_dir;
};

// Uniform integer noise of ARTSS src/randomField/UniformRandom.{h,cpp}:
// k ~ U{-steps..steps} from std::mt19937(seed), value k * step_size.
class UniformRandom {
 public:
    UniformRandom(real range, real step_size, size_t seed)
        : m_steps(static_cast<int>(range / step_size)), m_step_size(step_size), m_mt(seed),
          m_dist(-m_steps, m_steps) {}
    std::vector<real> random_field(size_t size) {
        std::vector<real> r(size);
        for (size_t i = 0; i < size; i++) r[i] = m_dist(m_mt) * m_step_size;
        return r;
    }

 private:
    int m_steps;
    real m_step_size;
    std::mt19937 m_mt;
    std::uniform_int_distribution<int> m_dist;
};

class GaussFunction : public ISourceFunction {
 public:
    GaussFunction(Runtime &rt, const settings::Gauss &s);
    void update_source(Field &out, real t_cur) override;
    void update_obstacle_change() override;
    void set_noise(std::unique_ptr<UniformRandom> noise, bool absolute) {
        m_noise = std::move(noise);
        m_absolute = absolute;
    }
    const Field &spatial_values() const { return m_spatial; }

 private:
    void create_spatial_values();
    Runtime &m_rt;
    settings::Gauss m_settings;
    Field m_spatial;
    std::unique_ptr<UniformRandom> m_noise;
    bool m_absolute = false;
    int m_param = -1;  // parameter slot of tanh(t / tau) in captured steps
};

class ZeroSource : public ISourceFunction {
 public:
    void update_source(Field &, real) override {}
    void update_obstacle_change() override {}
};

}  // namespace artss
