// Runtime of one scene: the device context built from the host geometry,
// and Field, the device array type the plugin interfaces pass around.
//
// Field keeps the interface of ARTSS src/field/Field.h:17-147 (set_value,
// copy_data, +=, *=, swap of data pointers) with the storage on the B200;
// every operation is a C-ABI call from include/artss_cuda.h.
#pragma once

#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/artss_cuda.h"
#include "geometry.h"
#include "settings.h"

namespace artss {

using real = double;

class cuda_error : public std::runtime_error {
 public:
    explicit cuda_error(const std::string &m) : std::runtime_error(m) {}
};

// throws cuda_error with the C-ABI's message when status != 0
void check(int status, const char *what);

class Runtime;

class Field {
 public:
    Field(Runtime &rt, int type, real value = 0.0, size_t level = 0);
    Field(const Field &) = delete;
    Field &operator=(const Field &) = delete;
    ~Field();

    int get_type() const { return m_type; }
    size_t get_level() const { return m_level; }
    size_t get_size() const { return m_size; }
    Runtime &runtime() const { return *m_rt; }

    void set_value(real val) const;
    void copy_data(const Field &other) const;
    Field &operator+=(real x);
    Field &operator+=(const Field &rhs);
    Field &operator*=(real x);
    static void swap(Field &a, Field &b) { std::swap(a.data, b.data); }

    std::vector<real> to_host() const;
    void from_host(const std::vector<real> &v);

    real *data = nullptr;  // device array, Nx*Ny*Nz of the level

 private:
    Runtime *m_rt;
    int m_type;
    size_t m_level;
    size_t m_size;
    real *m_owned = nullptr;
};

// Host transfers of one timestep overlapped with its computation (the
// context's second stream): inputs a solver reads late are uploaded there
// while the step runs and waited for at their first use (need); outputs are
// read back as soon as the solver has written them for the last time (done).
// Solvers without these calls get every input before and every output after
// the step.
class StepIO {
 public:
    struct In {
        Field *f;
        const real *host;
        int slot;
        bool waited;
    };
    struct Out {
        Field *f;
        real *host;
        bool sent;
    };
    explicit StepIO(artss_ctx *ctx) : m_ctx(ctx) {}
    void upload_late(Field &f, const real *host);  // on the second stream, after the uploads before it
    bool need(Field &f);                           // the step's later work waits for f's upload (true: f was uploaded)
    void add_output(Field &f, real *host) { m_out.push_back({&f, host, false}); }
    void done(Field &f);                           // f's value is final: read it back beside later work
    void finish();                                 // the rest, then the context waits for the transfers

 private:
    artss_ctx *m_ctx;
    std::vector<In> m_in;
    std::vector<Out> m_out;
};

class Runtime {
 public:
    Runtime(const settings::Settings &s, int device);
    ~Runtime();
    Runtime(const Runtime &) = delete;
    Runtime &operator=(const Runtime &) = delete;

    artss_ctx *ctx() const { return m_ctx; }
    const settings::Settings &settings() const { return m_settings; }
    const Geometry &geometry() const { return *m_geo; }
    const GridLevel &level(size_t l = 0) const { return m_geo->grid().level(l); }
    real dt() const { return m_settings.physical.dt; }

    // DomainController::apply_boundary
    void apply_boundary(Field &f) const;

    // transfers of the running step, when it runs through TimeIntegration::step_io
    StepIO *io = nullptr;

    // whole-step graphs (TimeIntegration): a captured step is replayed from
    // the third step on; values that change per step are set before each
    // replay by the providers plugins register here, into parameter slots
    bool graphs = false;
    std::vector<std::function<void(real)>> step_params;
    int next_param_slot = 0;
    bool capturing() const { return artss_graph_capturing(m_ctx) != 0; }

 private:
    settings::Settings m_settings;
    std::unique_ptr<Geometry> m_geo;
    artss_ctx *m_ctx = nullptr;
};

// Fills the descriptor the device context is created from.
artss_grid_desc grid_descriptor(const Geometry &g);

}  // namespace artss
