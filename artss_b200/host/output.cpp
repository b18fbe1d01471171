#include "output.h"

#include <cstdio>
#include <cstring>
#include <fstream>

namespace artss {

OutputWriter::OutputWriter(Runtime &rt) : m_rt(rt) {
    const GridLevel &g = rt.level(0);
    m_sight.assign(g.size(), 1.0f);
    for (Idx idx : rt.geometry().inner(0)) m_sight[(size_t) idx] = 0.0f;  // SolverController::update_sight
    m_thread = std::thread([this] { worker(); });
}

OutputWriter::~OutputWriter() {
    {
        std::lock_guard<std::mutex> lock(m_mutex);
        m_stop = true;
    }
    m_cv.notify_all();
    if (m_thread.joinable()) m_thread.join();
}

void OutputWriter::write_dat(const Field &f, const std::string &path) {
    const double *fields[1] = {f.data};
    int64_t ticket = -1;
    check(artss_readback(m_rt.ctx(), 1, fields, (int64_t) f.get_size(), &ticket), "write_dat");
    {
        std::lock_guard<std::mutex> lock(m_mutex);
        m_jobs.push_back({ticket, DAT, path, 1});
    }
    m_cv.notify_all();
}

void OutputWriter::write_vtk(const std::vector<const Field *> &fields, const std::string &path) {
    if (fields.size() != 8) throw std::invalid_argument("write_vtk: u, v, w, p, rhs, T, nu_t, S_T");
    std::vector<const double *> dev;
    for (const Field *f : fields) dev.push_back(f->data);
    int64_t ticket = -1;
    check(artss_readback(m_rt.ctx(), (int) dev.size(), dev.data(), (int64_t) fields[0]->get_size(), &ticket),
          "write_vtk");
    {
        std::lock_guard<std::mutex> lock(m_mutex);
        m_jobs.push_back({ticket, VTK, path, (int) dev.size()});
    }
    m_cv.notify_all();
}

void OutputWriter::wait() {
    std::unique_lock<std::mutex> lock(m_mutex);
    m_cv.wait(lock, [&] { return m_jobs.empty() && m_busy == 0; });
    if (!m_error.empty()) {
        std::string e;
        std::swap(e, m_error);
        throw std::runtime_error(e);
    }
}

void OutputWriter::worker() {
    for (;;) {
        Job job;
        {
            std::unique_lock<std::mutex> lock(m_mutex);
            m_cv.wait(lock, [&] { return m_stop || !m_jobs.empty(); });
            if (m_jobs.empty()) return;
            job = m_jobs.front();
            m_jobs.pop_front();
            m_busy++;
        }
        std::string err;
        std::vector<const double *> host((size_t) job.n);
        if (artss_readback_wait(m_rt.ctx(), job.ticket, host.data(), job.n) != ARTSS_OK) {
            err = std::string("read-back: ") + artss_last_error();
        } else {
            try {
                if (job.kind == DAT) {
                    // Analysis::write_file: `out << data[index] << std::endl`
                    std::ofstream out(job.path, std::ofstream::out);
                    const size_t n = m_rt.level(0).size();
                    for (size_t i = 0; i < n; i++) out << host[0][i] << std::endl;
                    if (!out) err = "cannot write " + job.path;
                } else {
                    write_vtk_file(job, host.data());
                }
            } catch (const std::exception &e) {
                err = e.what();
            }
            artss_readback_release(m_rt.ctx(), job.ticket);
        }
        {
            std::lock_guard<std::mutex> lock(m_mutex);
            if (!err.empty() && m_error.empty()) m_error = err;
            m_busy--;
        }
        m_cv.notify_all();
    }
}

namespace {

void put_be(std::FILE *f, float v) {
    unsigned char b[4];
    std::memcpy(b, &v, 4);
    const unsigned char r[4] = {b[3], b[2], b[1], b[0]};
    std::fwrite(r, 1, 4, f);
}

}  // namespace

// The legacy VTK layout of a rectilinear grid with cell data: the first cell
// scalar as SCALARS, the others as one FIELD block, big-endian floats, then an
// empty point-data section.
void OutputWriter::write_vtk_file(const Job &job, const double *const *host) {
    const GridLevel &g = m_rt.level(0);
    const auto &X1 = m_rt.geometry().grid().start_pd;
    const int Nx = (int) g.N[0], Ny = (int) g.N[1], Nz = (int) g.N[2];
    const double dx = g.spacing[0], dy = g.spacing[1], dz = g.spacing[2];
    const size_t n = g.size();
    std::string path = job.path;
    if (path.find(".vtk") == std::string::npos) path += ".vtk";
    std::FILE *f = std::fopen(path.c_str(), "w+");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::unique_ptr<std::FILE, int (*)(std::FILE *)> guard(f, std::fclose);
    // faces of the cells, then cell centres (VTKWriter.cpp:148-190)
    std::vector<float> xc(Nx + 1), yc(Ny + 1), zc(Nz + 1);
    for (int i = 0; i <= Nx; i++) xc[i] = static_cast<float>(X1[0] + (i - 1) * dx);
    for (int j = 0; j <= Ny; j++) yc[j] = static_cast<float>(X1[1] + (j - 1) * dy);
    for (int k = 0; k <= Nz; k++) zc[k] = static_cast<float>(X1[2] + (k - 1) * dz);
    std::fprintf(f, "# vtk DataFile Version 2.0\nWritten using VisIt writer\nBINARY\n");
    std::fprintf(f, "DATASET RECTILINEAR_GRID\nDIMENSIONS %d %d %d\n", Nx + 1, Ny + 1, Nz + 1);
    std::fprintf(f, "X_COORDINATES %d float\n", Nx + 1);
    for (float v : xc) put_be(f, v);
    std::fprintf(f, "Y_COORDINATES %d float\n", Ny + 1);
    for (float v : yc) put_be(f, v);
    std::fprintf(f, "Z_COORDINATES %d float\n", Nz + 1);
    for (float v : zc) put_be(f, v);
    std::fprintf(f, "CELL_DATA %d\n", (int) n);
    const float hx = static_cast<float>(0.5 * dx), hy = static_cast<float>(0.5 * dy), hz = static_cast<float>(0.5 * dz);
    auto centre = [&](int axis, size_t q) {
        const size_t k = q / ((size_t) Nx * Ny), j = (q / Nx) % Ny, i = q % Nx;
        return axis == 0 ? xc[i] + hx : axis == 1 ? yc[j] + hy : zc[k] + hz;
    };
    std::fprintf(f, "SCALARS x-coords float\nLOOKUP_TABLE default\n");
    for (size_t q = 0; q < n; q++) put_be(f, centre(0, q));
    std::fprintf(f, "FIELD FieldData 12\n");
    std::fprintf(f, "y-coords 1 %d float\n", (int) n);
    for (size_t q = 0; q < n; q++) put_be(f, centre(1, q));
    std::fprintf(f, "z-coords 1 %d float\n", (int) n);
    for (size_t q = 0; q < n; q++) put_be(f, centre(2, q));
    // host[]: u, v, w, p, rhs, T, nu_t, S_T
    const char *names[10] = {"x-velocity", "y-velocity", "z-velocity", "pressure", "divergence", "temperature",
                             "concentration", "sight", "turb_visc", "source_T"};
    const int src[10] = {0, 1, 2, 3, 4, 5, -1, -2, 6, 7};
    for (int v = 0; v < 10; v++) {
        std::fprintf(f, "%s 1 %d float\n", names[v], (int) n);
        for (size_t q = 0; q < n; q++)
            put_be(f, src[v] >= 0 ? static_cast<float>(host[src[v]][q]) : src[v] == -2 ? m_sight[q] : 0.0f);
    }
    // the (empty) point-data section that closes the file
    std::fprintf(f, "POINT_DATA %d\n", (Nx + 1) * (Ny + 1) * (Nz + 1));
    if (std::ferror(f)) throw std::runtime_error("cannot write " + path);
}

}  // namespace artss
