// TopVoxel reader (TOP3D_XL.m:458-586, CreateVoxelFEAmodel).  The file is a sequence of whitespace-
// separated tokens, read in the order the MATLAB reader reads them with fscanf:
//   <4 header words> <version word> 1.0
//   Resolution: nelx nely nelz
//   <2 words> flag                          (1: every solid voxel line also carries a density)
//   <2 words> numSolid   then numSolid lines "voxel [density]"        (1-based voxel indices)
//   Passive elements: n  then n voxel indices
//   Fixations: n         then n lines "node fx fy fz"                  (flags: 1 = DOF fixed)
//   Loads: n             then n lines "node Fx Fy Fz"
//   <2 words> k          then k blocks "Loads: n idx" + n lines        (further load cases)
// The literal words the MATLAB reader checks ("Resolution:", "Passive", "elements:", "Fixations:",
// "Loads:") are checked here too.  Host code only.
#include <array>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <map>
#include <new>

#include "topvoxel.hpp"

namespace t3d {

namespace {

struct Tokens {
    std::string text;
    size_t pos = 0;
    bool next(std::string* t) {
        while (pos < text.size() && std::isspace((unsigned char)text[pos])) ++pos;
        if (pos >= text.size()) return false;
        const size_t b = pos;
        while (pos < text.size() && !std::isspace((unsigned char)text[pos])) ++pos;
        *t = text.substr(b, pos - b);
        return true;
    }
};

class Reader {
  public:
    explicit Reader(std::string text) { tk_.text = std::move(text); }
    bool word(std::string* w, const char* what) {
        if (tk_.next(w)) return true;
        return fail(std::string("unexpected end of file reading ") + what);
    }
    bool expect(const char* lit) {
        std::string w;
        if (!word(&w, lit)) return false;
        if (w != lit) return fail(std::string("expected '") + lit + "', found '" + w + "'");
        return true;
    }
    bool skip(int n, const char* what) {
        std::string w;
        for (int i = 0; i < n; ++i)
            if (!word(&w, what)) return false;
        return true;
    }
    bool integer(int64_t* v, const char* what) {
        std::string w;
        if (!word(&w, what)) return false;
        char* end = nullptr;
        errno = 0;
        const long long x = std::strtoll(w.c_str(), &end, 10);
        if (errno || end == w.c_str() || *end) return fail(std::string("bad integer '") + w + "' for " + what);
        *v = x;
        return true;
    }
    bool real(double* v, const char* what) {
        std::string w;
        if (!word(&w, what)) return false;
        char* end = nullptr;
        errno = 0;
        const double x = std::strtod(w.c_str(), &end);
        if (errno || end == w.c_str() || *end || !std::isfinite(x))
            return fail(std::string("bad number '") + w + "' for " + what);
        *v = x;
        return true;
    }
    bool fail(const std::string& m) {
        if (err_.empty()) err_ = m;
        return false;
    }
    const std::string& error() const { return err_; }

  private:
    Tokens tk_;
    std::string err_;
};

// rows of (node, a, b, c) with 1-based nodes in [1, nn]; duplicates keep the first row; ascending
template <class T>
bool read_node_rows(Reader& rd, int64_t n, int64_t nn, const char* what, std::map<int64_t, std::array<T, 3>>* rows,
                    bool as_int) {
    for (int64_t i = 0; i < n; ++i) {
        int64_t node;
        if (!rd.integer(&node, what)) return false;
        if (node < 1 || node > nn) return rd.fail(std::string(what) + ": node index out of range");
        std::array<T, 3> v{};
        for (int c = 0; c < 3; ++c) {
            if (as_int) {
                int64_t f;
                if (!rd.integer(&f, what)) return false;
                v[c] = (T)f;
            } else {
                double f;
                if (!rd.real(&f, what)) return false;
                v[c] = (T)f;
            }
        }
        rows->emplace(node - 1, v);   // emplace keeps an existing key: the first occurrence wins
    }
    return true;
}

}  // namespace

static bool parse_topvoxel_impl(const char* path, VoxelModel* out, std::string* err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        *err = std::string("cannot open ") + path;
        return false;
    }
    Reader rd(std::string((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>()));
    VoxelModel m;
    auto done = [&](bool ok) {
        if (!ok) *err = "TopVoxel " + std::string(path) + ": " + rd.error();
        else *out = std::move(m);
        return ok;
    };
    double version = 0.0;
    if (!rd.skip(4, "file header") || !rd.skip(1, "version word") || !rd.real(&version, "version")) return done(false);
    if (version != 1.0) return done(rd.fail("unsupported format version"));
    int64_t nx, ny, nz;
    if (!rd.expect("Resolution:") || !rd.integer(&nx, "resolution") || !rd.integer(&ny, "resolution") ||
        !rd.integer(&nz, "resolution"))
        return done(false);
    // the grid of a context holds fewer than 2^31 / 3 nodes, so larger domains could not run anyway
    if (nx < 1 || ny < 1 || nz < 1 || nx > (1 << 20) || ny > (1 << 20) || nz > (1 << 20) ||
        nx * ny * nz > (int64_t)1 << 30)
        return done(rd.fail("resolution out of range"));
    m.nelx = (int)nx;
    m.nely = (int)ny;
    m.nelz = (int)nz;
    const int64_t nv = nx * ny * nz, nn = (nx + 1) * (ny + 1) * (nz + 1);
    int64_t flag, ns;
    if (!rd.skip(2, "density-values words") || !rd.integer(&flag, "density-values flag") ||
        !rd.skip(2, "solid-voxels words") || !rd.integer(&ns, "solid voxel count"))
        return done(false);
    if (ns < 1 || ns > nv) return done(rd.fail("solid voxel count out of range"));
    m.has_densities = flag != 0;
    m.voxel.assign((size_t)nv, 0);
    for (int64_t i = 0; i < ns; ++i) {
        int64_t k;
        double d;
        if (!rd.integer(&k, "solid voxel")) return done(false);
        if (m.has_densities && !rd.real(&d, "voxel density")) return done(false);
        if (k < 1 || k > nv) return done(rd.fail("solid voxel index out of range"));
        m.voxel[(size_t)(k - 1)] = 1;
    }
    for (uint8_t v : m.voxel) m.num_solid += v != 0;
    int64_t np;
    if (!rd.expect("Passive") || !rd.expect("elements:") || !rd.integer(&np, "passive element count"))
        return done(false);
    if (np < 0 || np > nv) return done(rd.fail("passive element count out of range"));
    for (int64_t i = 0; i < np; ++i) {
        int64_t k;
        if (!rd.integer(&k, "passive element")) return done(false);
        if (k < 1 || k > nv) return done(rd.fail("passive element index out of range"));
        if (m.voxel[(size_t)(k - 1)] == 0) return done(rd.fail("passive element is not a solid voxel"));
        m.voxel[(size_t)(k - 1)] = 2;
    }
    for (uint8_t v : m.voxel) m.num_passive += v == 2;
    int64_t nfix, nload, nadd;
    std::map<int64_t, std::array<int64_t, 3>> fix;
    std::map<int64_t, std::array<double, 3>> load;
    if (!rd.expect("Fixations:") || !rd.integer(&nfix, "fixation count")) return done(false);
    if (nfix < 0) return done(rd.fail("negative fixation count"));
    if (!read_node_rows(rd, nfix, nn, "fixations", &fix, true)) return done(false);
    if (!rd.expect("Loads:") || !rd.integer(&nload, "load count")) return done(false);
    if (nload < 0) return done(rd.fail("negative load count"));
    if (!read_node_rows(rd, nload, nn, "loads", &load, false)) return done(false);
    if (!rd.skip(2, "additional-loads words") || !rd.integer(&nadd, "additional load case count")) return done(false);
    if (nadd < 0) return done(rd.fail("negative additional load case count"));
    if (nadd > 64) return done(rd.fail("more than 64 additional load cases"));
    m.num_additional_loads = (int)nadd;
    m.case_node.resize((size_t)nadd);
    m.case_f.resize((size_t)nadd);
    std::vector<bool> seen((size_t)nadd, false);
    for (int64_t a = 0; a < nadd; ++a) {   // "Loads: n idx": case idx (2..K+1) of the loadingCond_ cell array
        int64_t n, idx;
        std::map<int64_t, std::array<double, 3>> extra;
        if (!rd.expect("Loads:") || !rd.integer(&n, "load count") || !rd.integer(&idx, "load case index"))
            return done(false);
        if (n < 0) return done(rd.fail("negative load count"));
        if (idx < 2 || idx > nadd + 1 || seen[(size_t)(idx - 2)])
            return done(rd.fail("load case indices must be 2..K+1, each once"));
        seen[(size_t)(idx - 2)] = true;
        if (!read_node_rows(rd, n, nn, "additional loads", &extra, false)) return done(false);
        for (const auto& kv : extra) {
            m.case_node[(size_t)(idx - 2)].push_back(kv.first);
            for (int c = 0; c < 3; ++c) m.case_f[(size_t)(idx - 2)].push_back(kv.second[c]);
        }
    }
    // A node loaded in any load case is not fixed: FEA_ApplyBoundaryCondition removes, case after case,
    // every fixation row whose node carries that case's load (setdiff, TOP3D_XL.m:1326-1331)
    for (const auto& kv : load) fix.erase(kv.first);
    for (const auto& nodes : m.case_node)
        for (int64_t nd : nodes) fix.erase(nd);
    for (const auto& kv : fix) {
        const uint8_t bits = (uint8_t)((kv.second[0] ? 1 : 0) | (kv.second[1] ? 2 : 0) | (kv.second[2] ? 4 : 0));
        if (!bits) continue;
        m.fix_node.push_back(kv.first);
        m.fix_bits.push_back(bits);
    }
    for (const auto& kv : load) {
        m.load_node.push_back(kv.first);
        for (int c = 0; c < 3; ++c) m.load_f.push_back(kv.second[c]);
    }
    return done(true);
}

bool parse_topvoxel(const char* path, VoxelModel* out, std::string* err) {
    try {
        return parse_topvoxel_impl(path, out, err);
    } catch (const std::bad_alloc&) {   // no exception crosses the C-ABI
        *err = std::string("TopVoxel ") + path + ": out of host memory";
        return false;
    }
}

}  // namespace t3d
