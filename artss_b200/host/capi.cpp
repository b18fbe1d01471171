// extern "C" surface of the host runtime (include/artss_host.h).
#include <cstring>
#include <cstdio>
#include "../../include/artss_host.h"

#include <map>
#include <memory>
#include <string>

#include "output.h"
#include "solvers.h"

using namespace artss;

struct artss_geom {
    settings::Settings settings;
    std::unique_ptr<Geometry> geo;
    std::map<std::pair<int, int>, std::vector<BcAssign>> programs;
};

struct artss_sim {
    std::unique_ptr<Runtime> rt;
    std::unique_ptr<SolverController> sc;
    std::unique_ptr<TimeIntegration> ti;
    std::unique_ptr<OutputWriter> out;  // created by the first write
    ~artss_sim() { out.reset(); }       // the writer's thread ends before the context goes
};

namespace {

thread_local std::string g_err;

template <typename F>
int guarded(F &&f) {
    try {
        return f();
    } catch (const config_error &e) {
        g_err = std::string("config error: ") + e.what();
        return ARTSS_ERR_ARG;
    } catch (const cuda_error &e) {
        g_err = e.what();
        return ARTSS_ERR_CUDA;
    } catch (const std::invalid_argument &e) {  // a pointer, name, size or file the call cannot use
        g_err = e.what();
        return ARTSS_ERR_ARG;
    } catch (const std::exception &e) {  // a call the simulation's state or kind does not allow
        g_err = e.what();
        return ARTSS_ERR_STATE;
    }
}

}  // namespace

extern "C" {

const char *artss_host_last_error(void) { return g_err.c_str(); }

int artss_geom_create(const char *xml_path, artss_geom **out) {
    return guarded([&] {
        if (!xml_path || !out) throw std::invalid_argument("null argument");
        auto g = std::make_unique<artss_geom>();
        g->settings = settings::parse_settings_file(xml_path);
        g->geo = std::make_unique<Geometry>(g->settings);
        *out = g.release();
        return ARTSS_OK;
    });
}

void artss_geom_destroy(artss_geom *g) { delete g; }

int artss_geom_levels(artss_geom *g) { return g ? (int) g->geo->levels() : -1; }

int artss_geom_obstacles(artss_geom *g) { return g ? (int) g->geo->obstacle_count() : -1; }

int artss_geom_list(artss_geom *g, const char *name, int level, const int64_t **data, int64_t *n) {
    return guarded([&] {
        if (!g || !name || !data || !n) throw std::invalid_argument("null argument");
        if (level < 0 || (size_t) level > g->geo->levels()) throw std::invalid_argument("level out of range");
        const std::string s(name);
        const IdxList *L = nullptr;
        if (s == "inner") L = &g->geo->inner(level);
        else if (s == "domain") L = &g->geo->domain(level);
        else if (s == "obst") L = &g->geo->obstacle_cells(level);
        else {
            for (int p = 0; p < kPatches && !L; p++) {
                if (s == std::string("bnd_") + kPatchNames[p]) L = &g->geo->boundary(level, p);
                for (size_t id = 0; id < g->geo->obstacle_count() && !L; id++)
                    if (s == "obst" + std::to_string(id) + "_" + kPatchNames[p]) L = &g->geo->obstacle(level, id).patch[p];
            }
        }
        if (!L) throw std::invalid_argument("unknown list '" + s + "'");
        *data = L->data();
        *n = (int64_t) L->size();
        return ARTSS_OK;
    });
}

int artss_geom_dims(artss_geom *g, int level, int64_t *dims3) {
    return guarded([&] {
        if (!g || !dims3 || level < 0 || (size_t) level > g->geo->levels()) throw std::invalid_argument("bad argument");
        const GridLevel &L = g->geo->grid().level(level);
        for (int a = 0; a < 3; a++) dims3[a] = (int64_t) L.N[a];
        return ARTSS_OK;
    });
}

int artss_geom_boundary_program(artss_geom *g, int level, int field_type, const artss_bc_assign **ops, int64_t *n) {
    return guarded([&] {
        if (!g || !ops || !n || level < 0 || (size_t) level > g->geo->levels() || field_type < 0 ||
            field_type >= kFieldTypesHost)
            throw std::invalid_argument("bad argument");
        auto key = std::make_pair(level, field_type);
        auto it = g->programs.find(key);
        if (it == g->programs.end())
            it = g->programs.emplace(key, g->geo->has_boundary(field_type)
                                              ? g->geo->boundary_program((size_t) level, field_type)
                                              : std::vector<BcAssign>{}).first;
        *ops = reinterpret_cast<const artss_bc_assign *>(it->second.data());
        *n = (int64_t) it->second.size();
        return ARTSS_OK;
    });
}

int artss_geom_grid_desc(artss_geom *g, artss_grid_desc *out) {
    return guarded([&] {
        if (!g || !out) throw std::invalid_argument("null argument");
        *out = grid_descriptor(*g->geo);
        return ARTSS_OK;
    });
}

int artss_sim_create(const char *xml_path, int device, artss_sim **out) {
    return guarded([&] {
        if (!xml_path || !out) throw std::invalid_argument("null argument");
        auto s = std::make_unique<artss_sim>();
        settings::Settings st = settings::parse_settings_file(xml_path);
        s->rt = std::make_unique<Runtime>(st, device);
        s->sc = std::make_unique<SolverController>(*s->rt);
        s->ti = std::make_unique<TimeIntegration>(*s->rt, *s->sc);
        check(artss_ctx_sync(s->rt->ctx()), "set-up");
        *out = s.release();
        return ARTSS_OK;
    });
}

void artss_sim_destroy(artss_sim *s) {
    if (!s) return;
    try {
        s->ti.reset();
        s->sc.reset();
        s->rt.reset();
    } catch (...) {
    }
    delete s;
}

int artss_sim_run(artss_sim *s, int64_t steps, int64_t *done) {
    return guarded([&] {
        if (!s) throw std::invalid_argument("null simulation");
        int64_t d = s->ti->run(steps);
        check(artss_ctx_sync(s->rt->ctx()), "run");
        if (done) *done = d;
        return ARTSS_OK;
    });
}

int artss_sim_step_io(artss_sim *s, int n_in, const char *const *in_names, const double *const *in_host, int n_out,
                      const char *const *out_names, double *const *out_host) {
    return guarded([&] {
        if (!s || n_in < 0 || n_out < 0 || (n_in && (!in_names || !in_host)) || (n_out && (!out_names || !out_host)))
            throw std::invalid_argument("bad step arguments");
        auto field = [&](const char *name) {
            Field *f = name ? s->sc->fields().by_name(name) : nullptr;
            if (!f) throw std::invalid_argument(std::string("unknown field ") + (name ? name : "(null)"));
            return f;
        };
        std::vector<std::pair<Field *, const real *>> in;
        std::vector<std::pair<Field *, real *>> out;
        for (int k = 0; k < n_in; k++) {
            if (!in_host[k]) throw std::invalid_argument("null input buffer");
            in.emplace_back(field(in_names[k]), in_host[k]);
        }
        for (int k = 0; k < n_out; k++) {
            if (!out_host[k]) throw std::invalid_argument("null output buffer");
            out.emplace_back(field(out_names[k]), out_host[k]);
        }
        s->ti->step_io(in, out);
        check(artss_ctx_sync(s->rt->ctx()), "step");
        return ARTSS_OK;
    });
}

int artss_sim_step_io_async(artss_sim *s, int n_in, const char *const *in_names, const double *const *in_host,
                            int n_out, const char *const *out_names, double *const *out_host) {
    return guarded([&] {
        if (!s || n_in < 0 || n_out < 0 || (n_in && (!in_names || !in_host)) || (n_out && (!out_names || !out_host)))
            throw std::invalid_argument("bad step arguments");
        auto field = [&](const char *name) {
            Field *f = name ? s->sc->fields().by_name(name) : nullptr;
            if (!f) throw std::invalid_argument(std::string("unknown field ") + (name ? name : "(null)"));
            return f;
        };
        std::vector<std::pair<Field *, const real *>> in;
        std::vector<std::pair<Field *, real *>> out;
        for (int k = 0; k < n_in; k++) {
            if (!in_host[k]) throw std::invalid_argument("null input buffer");
            in.emplace_back(field(in_names[k]), in_host[k]);
        }
        for (int k = 0; k < n_out; k++) {
            if (!out_host[k]) throw std::invalid_argument("null output buffer");
            out.emplace_back(field(out_names[k]), out_host[k]);
        }
        s->ti->step_io_async(in, out);
        return ARTSS_OK;
    });
}

int artss_sim_io_sync(artss_sim *s) {
    return guarded([&] {
        if (!s) throw std::invalid_argument("null argument");
        check(artss_io_sync(s->rt->ctx()), "io_sync");
        return ARTSS_OK;
    });
}

int artss_sim_set_graphs(artss_sim *s, int enable) {
    if (!s) return ARTSS_ERR_ARG;
    s->rt->graphs = enable != 0;
    return ARTSS_OK;
}

int64_t artss_sim_graph_steps(artss_sim *s) { return s ? s->ti->graph_steps : -1; }

int artss_sim_finished(artss_sim *s) { return s ? (s->ti->finished() ? 1 : 0) : -1; }
double artss_sim_time(artss_sim *s) { return s ? s->ti->time() : -1.0; }
int64_t artss_sim_step_index(artss_sim *s) { return s ? s->ti->step_index() : -1; }
int64_t artss_sim_inner_cells(artss_sim *s) { return s ? (int64_t) s->rt->geometry().inner(0).size() : -1; }
int64_t artss_sim_field_size(artss_sim *s) { return s ? (int64_t) s->rt->level(0).size() : -1; }
artss_ctx *artss_sim_context(artss_sim *s) { return s ? s->rt->ctx() : nullptr; }

double *artss_sim_field_device(artss_sim *s, const char *name) {
    if (!s || !name) return nullptr;
    Field *f = s->sc->fields().by_name(name);
    return f ? f->data : nullptr;
}

int artss_sim_get_field(artss_sim *s, const char *name, double *host, int64_t n) {
    return guarded([&] {
        if (!s || !name || !host) throw std::invalid_argument("null argument");
        Field *f = s->sc->fields().by_name(name);
        if (!f) throw std::invalid_argument(std::string("unknown field ") + name);
        if ((size_t) n != f->get_size()) throw std::invalid_argument("size mismatch");
        check(artss_download(s->rt->ctx(), host, f->data, n), "get_field");
        return ARTSS_OK;
    });
}

int artss_sim_set_field(artss_sim *s, const char *name, const double *host, int64_t n) {
    return guarded([&] {
        if (!s || !name || !host) throw std::invalid_argument("null argument");
        Field *f = s->sc->fields().by_name(name);
        if (!f) throw std::invalid_argument(std::string("unknown field ") + name);
        if ((size_t) n != f->get_size()) throw std::invalid_argument("size mismatch");
        check(artss_upload(s->rt->ctx(), f->data, host, n), "set_field");
        return ARTSS_OK;
    });
}

// Checkpoint file: "ARTSSCKP", u32 version 1, u32 number of fields, i64 step,
// f64 time, i64 Nx, Ny, Nz of level 0, then per field a 16-byte zero-padded
// name, an i64 count and count little-endian doubles.
static const char *const kCheckpointFields[] = {"u", "v", "w", "u0", "v0", "w0", "u_tmp", "v_tmp", "w_tmp", "nu_t",
                                                "kappa_t", "p", "p0", "rhs", "T", "T0", "T_tmp", "T_a", "f_x", "f_y",
                                                "f_z", "S_T"};

int artss_sim_save(artss_sim *s, const char *path) {
    return guarded([&] {
        if (!s || !path) throw std::invalid_argument("null argument");
        std::FILE *f = std::fopen(path, "wb");
        if (!f) throw std::runtime_error(std::string("cannot write ") + path);
        std::unique_ptr<std::FILE, int (*)(std::FILE *)> guard(f, std::fclose);
        const GridLevel &L0 = s->rt->level(0);
        const uint32_t version = 1, nf = (uint32_t) (sizeof(kCheckpointFields) / sizeof(*kCheckpointFields));
        const int64_t step = s->ti->step_index(), dims[3] = {(int64_t) L0.N[0], (int64_t) L0.N[1], (int64_t) L0.N[2]};
        const double t = s->ti->time();
        bool ok = std::fwrite("ARTSSCKP", 1, 8, f) == 8 && std::fwrite(&version, 4, 1, f) == 1 &&
                  std::fwrite(&nf, 4, 1, f) == 1 && std::fwrite(&step, 8, 1, f) == 1 && std::fwrite(&t, 8, 1, f) == 1 &&
                  std::fwrite(dims, 8, 3, f) == 3;
        std::vector<double> host;
        for (const char *name : kCheckpointFields) {
            Field *fld = s->sc->fields().by_name(name);
            const int64_t n = (int64_t) fld->get_size();
            host.resize((size_t) n);
            check(artss_download(s->rt->ctx(), host.data(), fld->data, n), "checkpoint");
            char tag[16] = {};
            std::strncpy(tag, name, sizeof(tag) - 1);
            ok = ok && std::fwrite(tag, 1, 16, f) == 16 && std::fwrite(&n, 8, 1, f) == 1 &&
                 std::fwrite(host.data(), 8, (size_t) n, f) == (size_t) n;
        }
        if (!ok) throw std::runtime_error(std::string("short write to ") + path);
        return ARTSS_OK;
    });
}

int artss_sim_restore(artss_sim *s, const char *path) {
    return guarded([&] {
        if (!s || !path) throw std::invalid_argument("null argument");
        std::FILE *f = std::fopen(path, "rb");
        if (!f) throw std::runtime_error(std::string("cannot read ") + path);
        std::unique_ptr<std::FILE, int (*)(std::FILE *)> guard(f, std::fclose);
        char magic[8];
        uint32_t version = 0, nf = 0;
        int64_t step = 0, dims[3] = {};
        double t = 0;
        if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "ARTSSCKP", 8) != 0 || std::fread(&version, 4, 1, f) != 1 ||
            version != 1 || std::fread(&nf, 4, 1, f) != 1 || std::fread(&step, 8, 1, f) != 1 ||
            std::fread(&t, 8, 1, f) != 1 || std::fread(dims, 8, 3, f) != 3)
            throw std::invalid_argument(std::string(path) + " is not an ARTSS checkpoint");
        const GridLevel &L0 = s->rt->level(0);
        if (dims[0] != (int64_t) L0.N[0] || dims[1] != (int64_t) L0.N[1] || dims[2] != (int64_t) L0.N[2])
            throw std::invalid_argument("checkpoint grid differs from the scene's");
        std::vector<double> host;
        for (uint32_t q = 0; q < nf; q++) {
            char tag[17] = {};
            int64_t n = 0;
            if (std::fread(tag, 1, 16, f) != 16 || std::fread(&n, 8, 1, f) != 1)
                throw std::invalid_argument("truncated checkpoint");
            Field *fld = s->sc->fields().by_name(tag);
            if (!fld || (size_t) n != fld->get_size()) throw std::invalid_argument(std::string("checkpoint field ") + tag);
            host.resize((size_t) n);
            if (std::fread(host.data(), 8, (size_t) n, f) != (size_t) n) throw std::invalid_argument("truncated checkpoint");
            check(artss_upload(s->rt->ctx(), fld->data, host.data(), n), "restore");
        }
        s->ti->set_step(step);
        return ARTSS_OK;
    });
}

int artss_sim_write_dat(artss_sim *s, const char *field, const char *path) {
    return guarded([&] {
        if (!s || !field || !path) throw std::invalid_argument("null argument");
        Field *f = s->sc->fields().by_name(field);
        if (!f) throw std::invalid_argument(std::string("unknown field ") + field);
        if (!s->out) s->out = std::make_unique<OutputWriter>(*s->rt);
        s->out->write_dat(*f, path);
        return ARTSS_OK;
    });
}

int artss_sim_write_vtk(artss_sim *s, const char *path) {
    return guarded([&] {
        if (!s || !path) throw std::invalid_argument("null argument");
        FieldController &fc = s->sc->fields();
        if (!s->out) s->out = std::make_unique<OutputWriter>(*s->rt);
        s->out->write_vtk({&fc.u, &fc.v, &fc.w, &fc.p, &fc.rhs, &fc.T, &fc.nu_t, &fc.S_T}, path);
        return ARTSS_OK;
    });
}

int artss_sim_output_wait(artss_sim *s) {
    return guarded([&] {
        if (!s) throw std::invalid_argument("null simulation");
        if (s->out) s->out->wait();
        return ARTSS_OK;
    });
}

int artss_sim_cfl(artss_sim *s, double *cfl) {
    return guarded([&] {
        if (!s || !cfl) throw std::invalid_argument("null argument");
        FieldController &fc = s->sc->fields();
        check(artss_cfl(s->rt->ctx(), fc.u.data, fc.v.data, fc.w.data, s->rt->dt(), cfl), "cfl");
        return ARTSS_OK;
    });
}

int artss_sim_last_stats(artss_sim *s, int64_t *diff_iters4, int64_t *mg_cycles, double *mg_residual) {
    return guarded([&] {
        if (!s) throw std::invalid_argument("null simulation");
        auto *ns = dynamic_cast<NSTempTurbSolver *>(&s->sc->solver());
        if (!ns) throw std::logic_error("statistics are kept by NSTempTurbSolver scenes");
        if (diff_iters4)
            for (int k = 0; k < 4; k++) diff_iters4[k] = ns->stats.diffusion_iterations[k];
        if (mg_cycles) *mg_cycles = ns->stats.pressure_cycles;
        if (mg_residual) *mg_residual = ns->stats.pressure_residual;
        return ARTSS_OK;
    });
}

int artss_sim_pressure(artss_sim *s, int first_step, int64_t *cycles, double *residual) {
    return guarded([&] {
        if (!s) throw std::invalid_argument("null simulation");
        auto *ps = dynamic_cast<PressureSolver *>(&s->sc->solver());
        if (!ps) throw std::logic_error("not a PressureSolver scene");
        const real dt = s->rt->dt();
        ps->pressure().pressure(s->sc->fields().p, s->sc->fields().rhs, first_step ? dt : 2 * dt, false);
        check(artss_ctx_sync(s->rt->ctx()), "pressure");
        if (cycles) *cycles = ps->pressure().last_cycles;
        if (residual) *residual = ps->pressure().last_residual;
        return ARTSS_OK;
    });
}

artss_mg *artss_sim_mg(artss_sim *s) {
    if (!s) return nullptr;
    if (auto *ps = dynamic_cast<PressureSolver *>(&s->sc->solver()))
        if (auto *mg = dynamic_cast<VCycleMG *>(&ps->pressure())) return mg->handle();
    return nullptr;
}

}  // extern "C"
