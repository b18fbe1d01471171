// Oracle driver for the reference serial build (test infrastructure only).
//
// Links the unmodified ARTSS translation units compiled by oracle/Makefile
// and reproduces the set-up of ARTSS src/main.cpp:62-85 and the benchmark
// branch of the time loop in src/TimeIntegration.cpp:86-145, then dumps
// full-precision fields and the multigrid index lists so that the B200 path
// can be checked against the reference bit for bit (lists) and to ~1e-16
// (fields).  Nothing under artss_b200/ links or runs this program; tests and
// the CPU-baseline leg of bench.py call it as the checker.
//
// Usage:
//   artss_ref_driver <file.xml> [--steps N] [--dump DIR] [--every K]
//                    [--lists] [--time] [--mg-rhs rhs.f64 --mg-rel-tol TOL]
//                    [--fields u,v,w,...]   (dump only these fields)
//                    [--vtk PREFIX] [--dat FIELD:PATH] [--cfl]
//                    (after the steps: VTKWriter::write_numerical to PREFIX.vtk,
//                     Analysis::write_file of one field, Analysis::calc_CFL printed)
//
// Dump layout (all little-endian, raw):
//   DIR/meta.txt                       grid sizes per level, dt, steps
//   DIR/step%05d_<field>.f64           Nx*Ny*Nz doubles of level 0
//   DIR/lists/<name>_L<level>.u64      size_t index lists per level
//
// Private members of Multigrid are reached by compiling this one file with
// `private`/`protected` mapped to `public`; class layout is unchanged.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <cmath>
#include <new>
#include <string>
#include <vector>
#include <fstream>
#include <sys/stat.h>
// Every standard header the reference headers use is included before the
// access-specifier remap below so that only ARTSS classes are affected.
#include <algorithm>
#include <array>
#include <cstddef>
#include <filesystem>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <optional>
#include <random>
#include <sstream>
#include <stdexcept>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <variant>

#define private public
#define protected public
#include "src/utility/settings/Settings.h"
#include "src/domain/DomainData.h"
#include "src/domain/DomainController.h"
#include "src/domain/Multigrid.h"
#include "src/solver/SolverController.h"
#include "src/field/FieldController.h"
#include "src/pressure/VCycleMG.h"
#include "src/solver/SolverSelection.h"
#include "src/solver/NSTempTurbSolver.h"
#include "src/source/GaussFunction.h"
#include "src/analysis/Analysis.h"
#include "src/analysis/Solution.h"
#include "src/visualisation/VTKWriter.h"
#undef private
#undef protected

// The reference allocates most fields with `new real[n]` and never
// initialises them (src/field/Field.cpp:12-25).  Serving every array
// allocation zero-filled makes a run deterministic; the B200 path likewise
// starts every field at zero.
void *operator new[](std::size_t n) {
    void *p = std::calloc(n ? n : 1, 1);
    if (!p) throw std::bad_alloc();
    return p;
}
void operator delete[](void *p) noexcept { std::free(p); }
void operator delete[](void *p, std::size_t) noexcept { std::free(p); }

namespace {

void make_dir(const std::string &d) { mkdir(d.c_str(), 0755); }

void write_raw(const std::string &path, const void *data, size_t bytes) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) { std::perror(path.c_str()); std::exit(2); }
    if (bytes && std::fwrite(data, 1, bytes, f) != bytes) { std::perror(path.c_str()); std::exit(2); }
    std::fclose(f);
}

void dump_list(const std::string &dir, const std::string &name, size_t level,
               const size_t *data, size_t count) {
    write_raw(dir + "/" + name + "_L" + std::to_string(level) + ".u64", data, count * sizeof(size_t));
}

void dump_lists(const std::string &dir) {
    const std::string ldir = dir + "/lists";
    make_dir(ldir);
    auto dc = DomainController::getInstance();
    Multigrid *mg = dc->m_multigrid;
    const size_t levels = DomainData::getInstance()->get_levels();
    for (size_t l = 0; l <= levels; l++) {
        const SingleJoinedList &in = mg->m_jl_domain_inner_list;
        dump_list(ldir, "inner", l, in.get_data() + in.get_first_index(l), in.get_slice_size(l));
        const SingleJoinedList &dl = mg->m_jl_domain_list;
        dump_list(ldir, "domain", l, dl.get_data() + dl.get_first_index(l), dl.get_slice_size(l));
        for (size_t p = 0; p < number_of_patches; p++) {
            SingleJoinedList *b = mg->m_jl_domain_boundary_list_patch_divided[p];
            dump_list(ldir, "bnd_" + patch_names[p], l, b->get_data() + b->get_first_index(l), b->get_slice_size(l));
        }
        if (mg->m_number_of_obstacle_objects > 0) {
            const SingleJoinedList &ol = mg->m_jl_obstacle_list;
            dump_list(ldir, "obst", l, ol.get_data() + ol.get_first_index(l), ol.get_slice_size(l));
            for (size_t id = 0; id < mg->m_number_of_obstacle_objects; id++) {
                for (size_t p = 0; p < number_of_patches; p++) {
                    MultipleJoinedList *m = mg->m_jl_obstacle_boundary_list_patch_divided[p];
                    dump_list(ldir, "obst" + std::to_string(id) + "_" + patch_names[p], l,
                              m->get_data() + m->get_first_index(l, id), m->get_slice_size(l, id));
                }
            }
        }
    }
}

struct NamedField { const char *name; Field *f; };

std::vector<NamedField> all_fields(FieldController *fc) {
    return {
        {"u", &fc->get_field_u()}, {"v", &fc->get_field_v()}, {"w", &fc->get_field_w()},
        {"p", &fc->get_field_p()}, {"T", &fc->get_field_T()}, {"nu_t", &fc->get_field_nu_t()},
        {"rhs", &fc->get_field_rhs()}, {"kappa_t", &fc->get_field_kappa()},
        {"S_T", &fc->get_field_source_T()}, {"f_x", &fc->get_field_force_x()},
        {"f_y", &fc->get_field_force_y()}, {"f_z", &fc->get_field_force_z()},
        {"T_a", &fc->get_field_T_ambient()},
    };
}

// comma-separated field names to dump; empty = all
std::string g_dump_only;

bool wanted(const char *name) {
    if (g_dump_only.empty()) return true;
    const std::string key = "," + g_dump_only + ",";
    return key.find("," + std::string(name) + ",") != std::string::npos;
}

void dump_fields(const std::string &dir, size_t step, FieldController *fc) {
    char prefix[64];
    std::snprintf(prefix, sizeof(prefix), "/step%05zu_", step);
    for (auto &nf : all_fields(fc)) {
        if (!wanted(nf.name)) continue;
        write_raw(dir + prefix + nf.name + ".f64", nf.f->data, nf.f->get_size() * sizeof(double));
    }
}

void write_meta(const std::string &dir, size_t steps_run) {
    auto dd = DomainData::getInstance();
    std::ofstream m(dir + "/meta.txt");
    m.precision(17);
    m << "levels " << dd->get_levels() << "\n";
    for (size_t l = 0; l <= dd->get_levels(); l++) {
        m << "level " << l << " Nx " << dd->get_number_of_cells(CoordinateAxis::X, l)
          << " Ny " << dd->get_number_of_cells(CoordinateAxis::Y, l)
          << " Nz " << dd->get_number_of_cells(CoordinateAxis::Z, l)
          << " nx " << dd->get_number_of_inner_cells(CoordinateAxis::X, l)
          << " ny " << dd->get_number_of_inner_cells(CoordinateAxis::Y, l)
          << " nz " << dd->get_number_of_inner_cells(CoordinateAxis::Z, l) << "\n";
    }
    m << "dt " << dd->get_physical_parameters().dt << "\n";
    m << "steps " << steps_run << "\n";
}

std::vector<double> read_f64(const std::string &path, size_t n) {
    std::vector<double> v(n);
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(v.data(), sizeof(double), n, f) != n) {
        std::fprintf(stderr, "cannot read %zu doubles from %s\n", n, path.c_str());
        std::exit(2);
    }
    std::fclose(f);
    return v;
}

// ||b - A p||_2 / ||b||_2 over the level-0 inner list, with A the 7-point
// Laplacian exactly as in VCycleMG::pressure (src/pressure/VCycleMG.cpp:186-194).
double relative_residual(const Field &p, const Field &b) {
    auto dd = DomainData::getInstance();
    auto dc = DomainController::getInstance();
    const size_t Nx = dd->get_Nx(), Ny = dd->get_Ny();
    const double rdx2 = 1. / (dd->get_dx() * dd->get_dx());
    const double rdy2 = 1. / (dd->get_dy() * dd->get_dy());
    const double rdz2 = 1. / (dd->get_dz() * dd->get_dz());
    const size_t n = dc->get_size_domain_inner_list_level_joined(0);
    const size_t *list = dc->get_domain_inner_list_level_joined();
    double sr = 0., sb = 0.;
    for (size_t j = 0; j < n; j++) {
        const size_t i = list[j];
        double r = b[i] - (rdx2 * (p[i - 1] - 2 * p[i] + p[i + 1])
                         + rdy2 * (p[i - Nx] - 2 * p[i] + p[i + Nx])
                         + rdz2 * (p[i - Nx * Ny] - 2 * p[i] + p[i + Nx * Ny]));
        sr += r * r;
        sb += b[i] * b[i];
    }
    return std::sqrt(sr) / std::sqrt(sb);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s file.xml [--steps N] [--dump DIR] [--every K] [--lists] [--time]"
                             " [--mg-rhs rhs.f64 --mg-rel-tol TOL --mg-max-cycles N] [--fields a,b,...]\n", argv[0]);
        return 1;
    }
    std::string xml = argv[1];
    long max_steps = -1;
    std::string dump_dir;
    long every = 1;
    bool lists = false, timing = false;
    std::string mg_rhs, vtk_prefix, dat_spec;
    bool print_cfl = false;
    double mg_rel_tol = 1e-8;
    long mg_max_cycles = 1000;
    for (int a = 2; a < argc; a++) {
        std::string k = argv[a];
        auto next = [&]() -> std::string {
            if (a + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", k.c_str()); std::exit(1); }
            return argv[++a];
        };
        if (k == "--steps") max_steps = std::stol(next());
        else if (k == "--dump") dump_dir = next();
        else if (k == "--every") every = std::stol(next());
        else if (k == "--lists") lists = true;
        else if (k == "--time") timing = true;
        else if (k == "--mg-rhs") mg_rhs = next();
        else if (k == "--mg-rel-tol") mg_rel_tol = std::stod(next());
        else if (k == "--mg-max-cycles") mg_max_cycles = std::stol(next());
        else if (k == "--fields") g_dump_only = next();
        else if (k == "--vtk") vtk_prefix = next();
        else if (k == "--dat") dat_spec = next();
        else if (k == "--cfl") print_cfl = true;
        else { std::fprintf(stderr, "unknown option %s\n", k.c_str()); return 1; }
    }
    if (!dump_dir.empty()) make_dir(dump_dir);

    try {
        auto t_setup0 = std::chrono::steady_clock::now();
        Settings::Settings settings = Settings::parse_settings(xml);
        size_t multigrid_level = 0;
        const auto &solver = settings.solver_parameters.description;
        if (solver.find("NS") != std::string::npos || solver == SolverTypes::PressureSolver) {
            multigrid_level = settings.solver_parameters.pressure.solver.n_level;
        }
        DomainData::init(settings.physical_parameters, settings.domain_parameters, multigrid_level);
        DomainController::init(settings);
        if (lists && !dump_dir.empty()) dump_lists(dump_dir);

        auto *sc = new SolverController(settings);
        FieldController *fc = sc->get_field_controller();
        auto t_setup1 = std::chrono::steady_clock::now();

        if (!mg_rhs.empty()) {
            // Pressure-only harness: plain reference V-cycles from p = 0 on a
            // caller-supplied RHS until ||b - A p|| / ||b|| <= tol.
            auto dd = DomainData::getInstance();
            Field &p = fc->get_field_p();
            Field &rhs = fc->get_field_rhs();
            auto v = read_f64(mg_rhs, rhs.get_size());
            for (size_t i = 0; i < rhs.get_size(); i++) rhs[i] = v[i];
            p.set_value(0.);
            DomainController::getInstance()->apply_boundary(p);
            IPressure *pres = nullptr;
            SolverSelection::set_pressure_solver(settings.solver_parameters.pressure, &pres);
            auto *mg = dynamic_cast<VCycleMG *>(pres);
            auto t0 = std::chrono::steady_clock::now();
            mg->UpdateInput(p, rhs, true);
            long cycles = 0;
            double rr = relative_residual(p, rhs);
            while (rr > mg_rel_tol && cycles < mg_max_cycles) {
                mg->VCycleMultigrid(p, true);
                cycles++;
                rr = relative_residual(p, rhs);
            }
            auto t1 = std::chrono::steady_clock::now();
            double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
            std::printf("{\"mg_cycles\": %ld, \"rel_res\": %.6e, \"ms\": %.3f, \"inner_cells\": %zu}\n",
                        cycles, rr, ms, DomainController::getInstance()->get_size_domain_inner_list_level_joined(0));
            if (!dump_dir.empty()) write_raw(dump_dir + "/mg_p.f64", p.data, p.get_size() * sizeof(double));
            (void) dd;
            delete pres;
            delete sc;
            return 0;
        }

        auto dd = DomainData::getInstance();
        const double dt = dd->get_physical_parameters().dt;
        const double t_end = dd->get_physical_parameters().t_end;
        if (!dump_dir.empty()) {
            dump_fields(dump_dir, 0, fc);
            // spatial part of the Gaussian heat source (GaussFunction.cpp:53-107)
            if (auto *ns = dynamic_cast<NSTempTurbSolver *>(sc->m_solver))
                if (auto *gf = dynamic_cast<GaussFunction *>(ns->m_source_function_temperature))
                    write_raw(dump_dir + "/gauss_spatial.f64", gf->m_field_spatial_values.data,
                              gf->m_field_spatial_values.get_size() * sizeof(double));
        }

        double t_cur = dt;
        long step = 1;
        std::vector<double> step_ms;
        auto loop0 = std::chrono::steady_clock::now();
        while (t_cur < t_end + dt / 2 && (max_steps < 0 || step <= max_steps)) {
            auto s0 = std::chrono::steady_clock::now();
            sc->solver_do_step(t_cur, false);
            sc->update_sources(t_cur, false);
            fc->update_data(false);
            auto s1 = std::chrono::steady_clock::now();
            step_ms.push_back(std::chrono::duration<double, std::milli>(s1 - s0).count());
            if (!dump_dir.empty() && (step % every == 0)) dump_fields(dump_dir, (size_t) step, fc);
            step++;
            t_cur = step * dt;
        }
        auto loop1 = std::chrono::steady_clock::now();
        const long steps_run = step - 1;
        if (!vtk_prefix.empty()) VTKWriter::write_numerical(*fc, vtk_prefix);
        if (!dat_spec.empty() || print_cfl) {
            Solution solution(settings.initial_conditions_parameters, settings.solver_parameters.solution);
            Analysis analysis(settings.solver_parameters.solution, settings.visualisation_parameters, solution);
            if (!dat_spec.empty()) {
                const size_t colon = dat_spec.find(':');
                const std::string name = dat_spec.substr(0, colon), path = dat_spec.substr(colon + 1);
                for (auto &nf : all_fields(fc))
                    if (name == nf.name) analysis.write_file(*nf.f, path);  // appends ".dat"
            }
            if (print_cfl)
                std::printf("{\"cfl\": %.17g}\n", analysis.calc_CFL(fc->get_field_u(), fc->get_field_v(),
                                                                     fc->get_field_w(), dt));
        }
        if (!dump_dir.empty()) write_meta(dump_dir, (size_t) steps_run);
        if (timing) {
            const size_t inner = DomainController::getInstance()->get_size_domain_inner_list_level_joined(0);
            double loop_ms = std::chrono::duration<double, std::milli>(loop1 - loop0).count();
            double steady = 0.;
            for (size_t s = 1; s < step_ms.size(); s++) steady += step_ms[s];
            std::printf("{\"step_ms\": [");
            for (size_t s = 0; s < step_ms.size(); s++) std::printf("%s%.3f", s ? ", " : "", step_ms[s]);
            std::printf("], ");
            std::printf("\"steps\": %ld, \"loop_ms\": %.3f, \"first_step_ms\": %.3f, \"steady_ms_per_step\": %.3f,"
                        " \"setup_ms\": %.3f, \"inner_cells\": %zu, \"cell_updates_per_s\": %.6e}\n",
                        steps_run, loop_ms, step_ms.empty() ? 0. : step_ms[0],
                        step_ms.size() > 1 ? steady / (double) (step_ms.size() - 1) : 0.,
                        std::chrono::duration<double, std::milli>(t_setup1 - t_setup0).count(),
                        inner, loop_ms > 0 ? (double) inner * (double) steps_run / (loop_ms * 1e-3) : 0.);
        }
        delete sc;
    } catch (const std::exception &ex) {
        std::fprintf(stderr, "reference error: %s\n", ex.what());
        return 3;
    }
    return 0;
}
