// The reference's text formats behind the C ABI (include/mlfma_b200.h):
// plane wave, dipoles, RWG mesh (vertices, faces, rwgs) and the solution
// file.  Each input line is parsed the way the reference's importers parse it
// (an istringstream per line that reads the values it needs and ignores the
// rest; a line without them, blank ones included, is an error), with the
// reference's messages: "Unable to find file" and "Unable to parse line".
//   importPlaneWave  src/fileio.h:8-27
//   importDipoles    src/fileio.h:110-131
//   importVertices, importTriangles, importRWG  src/fileio.h:134-202
//   Solver::printSols  src/solver.cpp:149-165
#include <complex>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mlfma_b200.h"

int mlfma_internal_fail(int code, const std::string& msg);

namespace {

// Reads every line of path; each must yield `count` values of type T.
template <class T>
int read_rows(const char* path, int count, std::vector<T>& out) {
    if (!path) return mlfma_internal_fail(MLFMA_ERR_ARG, "null path");
    std::ifstream in(path);
    if (!in) return mlfma_internal_fail(MLFMA_ERR_ARG, std::string("Unable to find file: ") + path);
    std::string line;
    long long row = 0;
    while (std::getline(in, line)) {
        ++row;
        std::istringstream iss(line);
        for (int k = 0; k < count; ++k) {
            T v{};
            if (!(iss >> v))
                return mlfma_internal_fail(MLFMA_ERR_ARG, std::string("Unable to parse line ") + std::to_string(row) +
                                                              " of " + path);
            out.push_back(v);
        }
    }
    return MLFMA_OK;
}

}  // namespace

extern "C" {

int mlfma_read_planewave(const char* path, mlfma_planewave* pw) {
    if (!pw) return mlfma_internal_fail(MLFMA_ERR_ARG, "null argument");
    if (!path) return mlfma_internal_fail(MLFMA_ERR_ARG, "null path");
    std::ifstream in(path);
    if (!in) return mlfma_internal_fail(MLFMA_ERR_ARG, std::string("Unable to find file: ") + path);
    std::string line;
    std::getline(in, line);  // only the first line is read
    std::istringstream iss(line);
    double v[8];
    for (double& x : v)
        if (!(iss >> x)) return mlfma_internal_fail(MLFMA_ERR_ARG, std::string("Unable to parse line 1 of ") + path);
    pw->amplitude = v[0];
    for (int k = 0; k < 3; ++k) {
        pw->pol[k] = v[1 + k];
        pw->khat[k] = v[4 + k];
    }
    pw->wavenum = v[7];
    return MLFMA_OK;
}

int mlfma_create_dipoles_from_file(const mlfma_config* cfg, const mlfma_planewave* pw, const char* path,
                                   mlfma_handle* out) {
    std::vector<double> a;
    const int rc = read_rows(path, 6, a);
    if (rc != MLFMA_OK) return rc;
    const int n = static_cast<int>(a.size() / 6);
    std::vector<double> pos(3 * static_cast<size_t>(n)), mom(3 * static_cast<size_t>(n));
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            pos[3 * static_cast<size_t>(i) + k] = a[6 * static_cast<size_t>(i) + k];
            mom[3 * static_cast<size_t>(i) + k] = a[6 * static_cast<size_t>(i) + 3 + k];
        }
    return mlfma_create_dipoles(cfg, pw, n, pos.data(), mom.data(), out);
}

int mlfma_create_rwg_from_files(const mlfma_config* cfg, const mlfma_planewave* pw, const char* vertices_path,
                                const char* faces_path, const char* rwgs_path, mlfma_handle* out) {
    std::vector<double> v;
    std::vector<int> f, r;
    int rc = read_rows(vertices_path, 3, v);
    if (rc == MLFMA_OK) rc = read_rows(faces_path, 3, f);
    if (rc == MLFMA_OK) rc = read_rows(rwgs_path, 4, r);
    if (rc != MLFMA_OK) return rc;
    return mlfma_create_rwg(cfg, pw, static_cast<int>(v.size() / 3), v.data(), static_cast<int>(f.size() / 3),
                            f.data(), static_cast<int>(r.size() / 4), r.data(), out);
}

int mlfma_write_solution(const char* path, int n, const double* x) {
    if (!path || (n > 0 && !x) || n < 0) return mlfma_internal_fail(MLFMA_ERR_ARG, "null argument");
    std::ofstream file(path);
    if (!file) return mlfma_internal_fail(MLFMA_ERR_ARG, std::string("Unable to open file: ") + path);
    file << std::setprecision(15) << std::scientific;
    for (int i = 0; i < n; ++i) file << std::complex<double>(x[2 * static_cast<size_t>(i)], x[2 * static_cast<size_t>(i) + 1]) << '\n';
    file.flush();
    if (!file) return mlfma_internal_fail(MLFMA_ERR_ARG, std::string("write failed: ") + path);
    return MLFMA_OK;
}

}  // extern "C"
