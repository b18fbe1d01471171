// Runtime of one scene: the device context built from the host geometry,
// and Field, the device array type the plugin interfaces pass around.
//
// Field keeps the interface of ARTSS src/field/Field.h:17-147 (set_value,
// copy_data, +=, *=, swap of data pointers) with the storage on the B200;
// every operation is a C-ABI call from include/artss_cuda.h.
#pragma once

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

 private:
    settings::Settings m_settings;
    std::unique_ptr<Geometry> m_geo;
    artss_ctx *m_ctx = nullptr;
};

// Fills the descriptor the device context is created from.
artss_grid_desc grid_descriptor(const Geometry &g);

}  // namespace artss
