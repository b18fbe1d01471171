// Output writers of the time loop, fed by snapshot read-backs
// (artss_readback): the values leave the device beside the following steps
// and a worker thread formats and writes the files, so the steps do not wait
// for the file system.
//  * write_dat: Analysis::write_file (src/analysis/Analysis.cpp:381-390), one
//    value per line in the default stream format, every cell of level 0;
//  * write_vtk: VTKWriter::write_numerical (src/visualisation/VTKWriter.cpp:60-
//    106): a legacy binary VTK rectilinear grid (big-endian floats) of the
//    level-0 cells with the cell centres, u, v, w, p, rhs, T, concentration,
//    the boundary "sight" (1 outside the inner cells) and nu_t, S_T.
#pragma once

#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "runtime.h"

namespace artss {

class OutputWriter {
 public:
    explicit OutputWriter(Runtime &rt);
    ~OutputWriter();
    OutputWriter(const OutputWriter &) = delete;
    OutputWriter &operator=(const OutputWriter &) = delete;

    void write_dat(const Field &f, const std::string &path);
    // u, v, w, p, rhs, T, nu_t, S_T (the concentration is written as 0)
    void write_vtk(const std::vector<const Field *> &fields, const std::string &path);
    // every write queued so far is on disk; rethrows the first failure
    void wait();

 private:
    enum Kind { DAT, VTK };
    struct Job {
        int64_t ticket;
        Kind kind;
        std::string path;
        int n;
    };
    void worker();
    void write_vtk_file(const Job &job, const double *const *host);
    Runtime &m_rt;
    std::vector<float> m_sight;  // 1 on every cell that is not inner
    std::mutex m_mutex;
    std::condition_variable m_cv;
    std::deque<Job> m_jobs;
    size_t m_busy = 0;
    bool m_stop = false;
    std::string m_error;
    std::thread m_thread;
};

}  // namespace artss
