#include "runtime.h"

static_assert(sizeof(artss::BcAssign) == sizeof(artss_bc_assign), "boundary assignment layout");

namespace artss {

void check(int status, const char *what) {
    if (status != ARTSS_OK) throw cuda_error(std::string(what) + ": " + artss_last_error());
}

artss_grid_desc grid_descriptor(const Geometry &g) {
    artss_grid_desc d{};
    d.n_levels = (int32_t) g.levels();
    if (g.levels() > ARTSS_MAX_LEVEL) throw config_error("more multigrid levels than the library supports");
    for (size_t l = 0; l <= g.levels(); l++) {
        const GridLevel &L = g.grid().level(l);
        d.Nx[l] = (int64_t) L.N[0];
        d.Ny[l] = (int64_t) L.N[1];
        d.Nz[l] = (int64_t) L.N[2];
        d.i1[l] = (int64_t) L.cd_start[0];
        d.i2[l] = (int64_t) L.cd_end[0];
        d.j1[l] = (int64_t) L.cd_start[1];
        d.j2[l] = (int64_t) L.cd_end[1];
        d.k1[l] = (int64_t) L.cd_start[2];
        d.k2[l] = (int64_t) L.cd_end[2];
        d.dx[l] = L.spacing[0];
        d.dy[l] = L.spacing[1];
        d.dz[l] = L.spacing[2];
    }
    return d;
}

Runtime::Runtime(const settings::Settings &s, int device) : m_settings(s) {
    m_geo = std::make_unique<Geometry>(m_settings);
    artss_grid_desc desc = grid_descriptor(*m_geo);
    check(artss_ctx_create(&desc, device, &m_ctx), "create device context");
    try {
        for (size_t l = 0; l <= m_geo->levels(); l++) {
            const IdxList &in = m_geo->inner(l);
            const IdxList &dl = m_geo->domain(l);
            check(artss_set_cell_lists(m_ctx, (int) l, in.data(), (int64_t) in.size(), dl.data(), (int64_t) dl.size()),
                  "upload cell lists");
            for (int ft = 0; ft < kFieldTypesHost; ft++) {
                if (!m_geo->has_boundary(ft)) continue;
                std::vector<BcAssign> ops = m_geo->boundary_program(l, ft);
                check(artss_set_boundary_program(m_ctx, (int) l, ft,
                                                 reinterpret_cast<const artss_bc_assign *>(ops.data()),
                                                 (int64_t) ops.size()),
                      "upload boundary program");
            }
        }
    } catch (...) {
        artss_ctx_destroy(m_ctx);
        m_ctx = nullptr;
        throw;
    }
}

Runtime::~Runtime() {
    if (m_ctx) artss_ctx_destroy(m_ctx);
}

void Runtime::apply_boundary(Field &f) const {
    check(artss_apply_boundary(m_ctx, f.data, (int) f.get_level(), f.get_type()), "apply_boundary");
}

Field::Field(Runtime &rt, int type, real value, size_t level)
    : m_rt(&rt), m_type(type), m_level(level), m_size(rt.level(level).size()) {
    check(artss_field_alloc(rt.ctx(), (int) level, &m_owned), "allocate field");
    data = m_owned;
    if (value != 0.0) set_value(value);
}

Field::~Field() {
    // data may have been swapped with another Field; the owned pointer is freed
    if (m_owned) artss_field_free(m_rt->ctx(), m_owned);
}

void Field::set_value(real val) const { check(artss_fill(m_rt->ctx(), data, (int) m_level, val), "set_value"); }

void Field::copy_data(const Field &other) const {
    check(artss_copy(m_rt->ctx(), data, other.data, (int) m_level), "copy_data");
}

Field &Field::operator+=(real x) {
    check(artss_add_scalar(m_rt->ctx(), data, x, (int) m_level), "operator+=");
    return *this;
}

Field &Field::operator+=(const Field &rhs) {
    check(artss_add_field(m_rt->ctx(), data, rhs.data, (int) m_level), "operator+=");
    return *this;
}

Field &Field::operator*=(real x) {
    check(artss_scale(m_rt->ctx(), data, x, (int) m_level), "operator*=");
    return *this;
}

std::vector<real> Field::to_host() const {
    std::vector<real> v(m_size);
    check(artss_download(m_rt->ctx(), v.data(), data, (int64_t) m_size), "download field");
    return v;
}

void Field::from_host(const std::vector<real> &v) {
    if (v.size() != m_size) throw std::invalid_argument("field size mismatch");
    check(artss_upload(m_rt->ctx(), data, v.data(), (int64_t) m_size), "upload field");
}

}  // namespace artss

namespace artss {

void StepIO::upload_late(Field &f, const real *host) {
    const int slot = (int) m_in.size();
    if (slot >= 8) throw std::invalid_argument("at most 8 inputs are uploaded during a step");
    check(artss_copy_upload(m_ctx, slot, f.data, host, (int64_t) f.get_size()), "upload");
    m_in.push_back({&f, host, slot, false});
}

bool StepIO::need(Field &f) {
    bool found = false;
    for (In &i : m_in)
        if (i.f == &f && !i.waited) {
            check(artss_copy_wait(m_ctx, i.slot), "upload wait");
            i.waited = true;
            found = true;
        }
    return found;
}

void StepIO::done(Field &f) {
    for (Out &o : m_out)
        if (o.f == &f && !o.sent) {
            check(artss_copy_download(m_ctx, o.host, f.data, (int64_t) f.get_size()), "download");
            o.sent = true;
        }
}

void StepIO::finish() {
    for (In &i : m_in)
        if (!i.waited) need(*i.f);
    for (Out &o : m_out)
        if (!o.sent) done(*o.f);
    check(artss_copy_join(m_ctx), "transfers");
}

}  // namespace artss
