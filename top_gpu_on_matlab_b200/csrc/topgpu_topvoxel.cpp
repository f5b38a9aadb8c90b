// topgpu_topvoxel.cpp -- .TopVoxel model files (format version 1.0): the
// file branch of CreateVoxelFEAmodel (TOP_GPU.m:416-496).
//
// The file is a stream of whitespace-separated tokens read in a fixed order:
//   4 header words, 1 word + version number (1.0),
//   "Resolution:" nelx nely nelz,
//   2 words + density flag, 2 words + number of solid voxels,
//   the solid voxels (1-based linear indices of the nely x nelx x nelz grid,
//   y fastest), each followed by its density when the flag is set,
//   "Passive" "elements:" count + element indices (same numbering),
//   "Fixations:" count + rows (node, fixX, fixY, fixZ),
//   "Loads:" count + rows (node, fx, fy, fz)       -- load case 1,
//   2 words + number of additional load blocks, each
//   "Loads:" count case + rows                      -- load case `case`.
// Node numbers refer to the (nely+1) x (nelx+1) x (nelz+1) node grid of the
// file.  After the voxel discretisation pads the grid (top_mesh_create), the
// fixations and loads keep one row per node (first occurrence, ascending),
// move to the padded node grid (AdaptBCExternalMdl, TOP_GPU.m:1743-1793) and
// to the compact node numbering (nodMapForward); passive elements likewise
// (AdaptPassiveElementsExternalMdl, 1795-1813, then eleMapForward).  Load
// cases are weighted equally (objWeightingList_).  Every non-empty load case
// is moved to the compact numbering (the reference does so only when case 1
// is not empty, TOP_GPU.m:483, and leaves the others in file numbering).
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "topgpu_internal.h"

using topgpu::MeshLevel;
using topgpu::set_error;

namespace {

constexpr const char *kFormatError = "Incompatible Mesh Data Format!";   // TOP_GPU.m:423 & co.

// whitespace-separated tokens scanned in place in the file's bytes (the
// buffer is NUL-terminated, so strtoll / strtod stop at a token's end)
struct Tokens {
    std::string buf;
    size_t i = 0;
    static bool ws(char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == '\v' || c == '\f'; }
    bool next(const char *&b, const char *&e)
    {
        while (i < buf.size() && ws(buf[i])) ++i;
        if (i >= buf.size()) return false;
        size_t j = i;
        while (j < buf.size() && !ws(buf[j])) ++j;
        b = buf.data() + i;
        e = buf.data() + j;
        i = j;
        return true;
    }
    bool skip(int n)
    {
        const char *b, *e;
        for (int k = 0; k < n; ++k)
            if (!next(b, e)) return false;
        return true;
    }
    // an upper bound on the tokens left (each takes a byte and a separator)
    size_t left() const { return (buf.size() - i + 1) / 2; }
    bool expect(const char *w)
    {
        const char *b, *e;
        return next(b, e) && size_t(e - b) == std::strlen(w) && std::memcmp(b, w, size_t(e - b)) == 0;
    }
    bool integer(int64_t &v)
    {
        const char *b, *e;
        if (!next(b, e)) return false;
        char *end = nullptr;
        errno = 0;
        const long long r = std::strtoll(b, &end, 10);
        if (errno || end != e) return false;
        v = r;
        return true;
    }
    bool real(double &v)
    {
        const char *b, *e;
        if (!next(b, e)) return false;
        char *end = nullptr;
        v = std::strtod(b, &end);
        return end == e;
    }
};

struct BcRow { int64_t node; double v[3]; size_t ord; };

// one row per node, first occurrence, ascending node (unique, TOP_GPU.m:468-470)
void unique_sorted(std::vector<BcRow> &r)
{
    for (size_t k = 0; k < r.size(); ++k) r[k].ord = k;
    std::sort(r.begin(), r.end(), [](const BcRow &a, const BcRow &b) { return a.node != b.node ? a.node < b.node : a.ord < b.ord; });
    size_t n = 0;
    for (size_t k = 0; k < r.size(); ++k)
        if (n == 0 || r[k].node != r[n - 1].node) r[n++] = r[k];
    r.resize(n);
}

// 1-based node of the file's node grid -> 1-based compact node of the padded
// mesh (0 when the node belongs to no solid voxel)
int64_t node_to_compact(const MeshLevel &L, int nely, int nelx, int64_t node)
{
    const int64_t g = node - 1, ny = nely + 1, nx = nelx + 1;
    const int64_t y = g % ny, x = (g / ny) % nx, z = g / (ny * nx);
    const int64_t py = L.resY + 1, px = L.resX + 1;
    return L.nodMapForward[(size_t)(y + py * (x + px * z))];
}

int64_t element_to_compact(const MeshLevel &L, int nely, int nelx, int64_t ele)
{
    const int64_t g = ele - 1;
    const int64_t y = g % nely, x = (g / nely) % nelx, z = g / ((int64_t)nely * nelx);
    return L.eleMapForward[(size_t)(y + (int64_t)L.resY * (x + (int64_t)L.resX * z))];
}

int fail(const char *what)
{
    set_error("top_mesh_create_from_topvoxel: %s", what);
    return TOP_ERR_ARGS;
}

}  // namespace

static int create_from_topvoxel(const char *path, int control, double nu, top_mesh **out)
{
    if (!path || !out || control < 1) return fail("bad arguments");
    *out = nullptr;
    Tokens tk;
    {
        std::FILE *f = std::fopen(path, "rb");
        if (!f) {
            set_error("top_mesh_create_from_topvoxel: cannot open '%s'", path);
            return TOP_ERR_ARGS;
        }
        char chunk[1 << 16];
        size_t n;
        while ((n = std::fread(chunk, 1, sizeof chunk, f)) > 0) tk.buf.append(chunk, n);
        std::fclose(f);
    }
    double version = 0;
    if (!tk.skip(4) || !tk.skip(1) || !tk.real(version)) return fail(kFormatError);
    if (version != 1.0) return fail("Unsupported Data! (format version other than 1.0)");   // TOP_GPU.m:463-464
    int64_t nelx = 0, nely = 0, nelz = 0;
    if (!tk.expect("Resolution:") || !tk.integer(nelx) || !tk.integer(nely) || !tk.integer(nelz)) return fail(kFormatError);
    if (nelx < 1 || nely < 1 || nelz < 1 || nelx > 65536 || nely > 65536 || nelz > 65536 ||
        nelx * nely * nelz > (int64_t(1) << 31))
        return fail("bad resolution");
    const int64_t NV = nelx * nely * nelz, NN = (nelx + 1) * (nely + 1) * (nelz + 1);
    int64_t withDensity = 0, nSolid = 0;
    if (!tk.skip(2) || !tk.integer(withDensity) || !tk.skip(2) || !tk.integer(nSolid) || nSolid < 0)
        return fail(kFormatError);
    std::vector<uint8_t> mask((size_t)NV, 0);
    std::vector<double> density;
    for (int64_t k = 0; k < nSolid; ++k) {
        int64_t v = 0;
        if (!tk.integer(v)) return fail(kFormatError);
        if (v < 1 || v > NV) return fail("solid voxel index outside the resolution");
        mask[(size_t)(v - 1)] = 1;
        if (withDensity) {
            double d = 0;
            if (!tk.real(d)) return fail(kFormatError);
            density.push_back(d);
        }
    }
    int64_t nPassive = 0;
    if (!tk.expect("Passive") || !tk.expect("elements:") || !tk.integer(nPassive) || nPassive < 0 ||
        (uint64_t)nPassive > tk.left())
        return fail(kFormatError);
    std::vector<int64_t> passive((size_t)nPassive);
    for (auto &p : passive) {
        if (!tk.integer(p)) return fail(kFormatError);
        if (p < 1 || p > NV) return fail("passive element index outside the resolution");
    }
    int64_t nFix = 0;
    if (!tk.expect("Fixations:") || !tk.integer(nFix) || nFix < 0 || (uint64_t)nFix > tk.left() / 4) return fail(kFormatError);
    std::vector<BcRow> fix((size_t)nFix);
    for (auto &r : fix) {
        int64_t c[3];
        if (!tk.integer(r.node) || !tk.integer(c[0]) || !tk.integer(c[1]) || !tk.integer(c[2])) return fail(kFormatError);
        if (r.node < 1 || r.node > NN) return fail("fixed node outside the node grid");
        for (int q = 0; q < 3; ++q) r.v[q] = double(c[q]);
    }
    auto read_loads = [&](int64_t n, std::vector<BcRow> &rows) -> bool {
        if ((uint64_t)n > tk.left() / 4) return false;
        rows.resize((size_t)n);
        for (auto &r : rows) {
            if (!tk.integer(r.node) || !tk.real(r.v[0]) || !tk.real(r.v[1]) || !tk.real(r.v[2])) return false;
            if (r.node < 1 || r.node > NN) return false;
        }
        return true;
    };
    std::vector<std::vector<BcRow>> loads(1);
    int64_t nLoad = 0;
    if (!tk.expect("Loads:") || !tk.integer(nLoad) || nLoad < 0 || !read_loads(nLoad, loads[0])) return fail(kFormatError);
    int64_t nMore = 0;
    if (!tk.skip(2) || !tk.integer(nMore) || nMore < 0) return fail(kFormatError);
    for (int64_t a = 0; a < nMore; ++a) {
        int64_t n = 0, idx = 0;
        if (!tk.expect("Loads:") || !tk.integer(n) || n < 0 || !tk.integer(idx) || idx < 1 || idx > 4096) return fail(kFormatError);
        if ((size_t)idx > loads.size()) loads.resize((size_t)idx);
        if (!read_loads(n, loads[(size_t)idx - 1])) return fail(kFormatError);
    }

    top_mesh *m = nullptr;
    int st = top_mesh_create(mask.data(), (int)nely, (int)nelx, (int)nelz, control, nu, 1.0, 0, &m);
    if (st != TOP_OK) return st;
    const MeshLevel &L = m->L[0];
    std::vector<double> fixRows;
    unique_sorted(fix);
    for (const BcRow &r : fix) {
        const int64_t c = node_to_compact(L, (int)nely, (int)nelx, r.node);
        if (!c) {
            top_mesh_destroy(m);
            set_error("top_mesh_create_from_topvoxel: fixed node %lld touches no solid voxel", (long long)r.node);
            return TOP_ERR_ARGS;
        }
        fixRows.insert(fixRows.end(), {double(c), r.v[0], r.v[1], r.v[2]});
    }
    std::vector<std::vector<double>> loadRows(loads.size());
    std::vector<int64_t> nRows(loads.size());
    std::vector<const double *> ptrs(loads.size());
    for (size_t k = 0; k < loads.size(); ++k) {
        unique_sorted(loads[k]);
        for (const BcRow &r : loads[k]) {
            const int64_t c = node_to_compact(L, (int)nely, (int)nelx, r.node);
            if (!c) {
                top_mesh_destroy(m);
                set_error("top_mesh_create_from_topvoxel: loaded node %lld touches no solid voxel", (long long)r.node);
                return TOP_ERR_ARGS;
            }
            loadRows[k].insert(loadRows[k].end(), {double(c), r.v[0], r.v[1], r.v[2]});
        }
        nRows[k] = (int64_t)loads[k].size();
        ptrs[k] = loadRows[k].data();
    }
    st = top_mesh_apply_bc(m, (int64_t)fix.size(), fixRows.data(), (int)loads.size(), nRows.data(), ptrs.data(), nullptr);
    if (st != TOP_OK) { top_mesh_destroy(m); return st; }
    std::sort(passive.begin(), passive.end());
    passive.erase(std::unique(passive.begin(), passive.end()), passive.end());
    for (int64_t p : passive) {
        const int64_t c = element_to_compact(L, (int)nely, (int)nelx, p);
        if (!c) {
            top_mesh_destroy(m);
            set_error("top_mesh_create_from_topvoxel: passive element %lld is not a solid voxel", (long long)p);
            return TOP_ERR_ARGS;
        }
        m->passiveElements.push_back((int32_t)c);
    }
    m->densityLayout = std::move(density);
    *out = m;
    return TOP_OK;
}

extern "C" int top_mesh_create_from_topvoxel(const char *path, int control, double nu, top_mesh **out)
{
    try {
        return create_from_topvoxel(path, control, nu, out);
    } catch (const std::bad_alloc &) {
        set_error("top_mesh_create_from_topvoxel: out of host memory");
        return TOP_ERR_NOMEM;
    }
}
