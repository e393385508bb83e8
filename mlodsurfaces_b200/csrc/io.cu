// io.cu -- point-set and parameter files (host code).
//
// Pn::load / Pn::save / Pn::normalize (sources/apss/Pn.cpp:102-290): .pn is
// raw float32 (x, y, z, nx, ny, nz) records; .ply is read for the vertex
// element's x, y, z and (optionally) nx, ny, nz properties in any of the PLY
// encodings and scalar types, and written as binary little endian floats the
// way Pn::save does.  normalize moves the cloud to its mean and divides by the
// largest coordinate of its (slightly widened) box, in float, in the same
// order of operations.  The .params file (scene::loadParameters,
// scene.cpp:1183-1250) is a packed sequence of fields, read and written here
// field by field.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "mlods_internal.cuh"

struct mlods_cloud_s {
    std::vector<float> pos, nrm;
    float offset[3] = {0.f, 0.f, 0.f};
    float norme = 1.f;
    bool has_normals = false;
};

namespace mlods
{
namespace
{
bool ends_with(const std::string& s, const std::string& e)
{
    return s.size() >= e.size() && s.compare(s.size() - e.size(), e.size(), e) == 0;
}

enum class PlyFormat { Ascii, Le, Be };

struct PlyProp {
    std::string name;
    int size = 0;        // bytes of a scalar
    char kind = 'f';     // 'f' float, 'i' signed, 'u' unsigned
    bool list = false;
    int count_size = 0;  // list count type
    char count_kind = 'u';
};

struct PlyElement {
    std::string name;
    int64_t count = 0;
    std::vector<PlyProp> props;
};

bool scalar_type(const std::string& t, int& size, char& kind)
{
    static const struct {
        const char* name;
        int size;
        char kind;
    } types[] = {{"char", 1, 'i'},   {"int8", 1, 'i'},    {"uchar", 1, 'u'},  {"uint8", 1, 'u'},
                 {"short", 2, 'i'},  {"int16", 2, 'i'},   {"ushort", 2, 'u'}, {"uint16", 2, 'u'},
                 {"int", 4, 'i'},    {"int32", 4, 'i'},   {"uint", 4, 'u'},   {"uint32", 4, 'u'},
                 {"float", 4, 'f'},  {"float32", 4, 'f'}, {"double", 8, 'f'}, {"float64", 8, 'f'}};
    for (const auto& x : types)
        if (t == x.name) {
            size = x.size;
            kind = x.kind;
            return true;
        }
    return false;
}

double decode(const unsigned char* p, int size, char kind, bool swap)
{
    unsigned char b[8];
    for (int i = 0; i < size; ++i) b[i] = swap ? p[size - 1 - i] : p[i];
    switch (kind) {
    case 'f':
        if (size == 4) {
            float f;
            std::memcpy(&f, b, 4);
            return f;
        } else {
            double d;
            std::memcpy(&d, b, 8);
            return d;
        }
    case 'i':
        if (size == 1) return double(int8_t(b[0]));
        if (size == 2) {
            int16_t v;
            std::memcpy(&v, b, 2);
            return v;
        }
        {
            int32_t v;
            std::memcpy(&v, b, 4);
            return v;
        }
    default:
        if (size == 1) return b[0];
        if (size == 2) {
            uint16_t v;
            std::memcpy(&v, b, 2);
            return v;
        }
        {
            uint32_t v;
            std::memcpy(&v, b, 4);
            return v;
        }
    }
}

int read_ply(const std::string& path, mlods_cloud_s& c)
{
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        set_last_error("ply: cannot open %s", path.c_str());
        return MLODS_ERR_INVALID;
    }
    std::string line;
    if (!std::getline(in, line) || line.rfind("ply", 0) != 0) {
        set_last_error("ply: %s is not a PLY file", path.c_str());
        return MLODS_ERR_INVALID;
    }
    PlyFormat fmt = PlyFormat::Ascii;
    std::vector<PlyElement> elems;
    bool header_done = false;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::istringstream ss(line);
        std::string w;
        ss >> w;
        if (w == "format") {
            std::string f;
            ss >> f;
            if (f == "ascii") fmt = PlyFormat::Ascii;
            else if (f == "binary_little_endian") fmt = PlyFormat::Le;
            else if (f == "binary_big_endian") fmt = PlyFormat::Be;
            else {
                set_last_error("ply: unknown format %s", f.c_str());
                return MLODS_ERR_INVALID;
            }
        } else if (w == "element") {
            PlyElement e;
            ss >> e.name >> e.count;
            if (e.count < 0) {
                set_last_error("ply: bad element count");
                return MLODS_ERR_INVALID;
            }
            elems.push_back(e);
        } else if (w == "property") {
            if (elems.empty()) {
                set_last_error("ply: property before any element");
                return MLODS_ERR_INVALID;
            }
            PlyProp p;
            std::string t;
            ss >> t;
            if (t == "list") {
                std::string ct, it;
                ss >> ct >> it >> p.name;
                p.list = true;
                if (!scalar_type(ct, p.count_size, p.count_kind) || !scalar_type(it, p.size, p.kind)) {
                    set_last_error("ply: unknown list type %s %s", ct.c_str(), it.c_str());
                    return MLODS_ERR_INVALID;
                }
            } else {
                ss >> p.name;
                if (!scalar_type(t, p.size, p.kind)) {
                    set_last_error("ply: unknown property type %s", t.c_str());
                    return MLODS_ERR_INVALID;
                }
            }
            elems.back().props.push_back(p);
        } else if (w == "end_header") {
            header_done = true;
            break;
        }
    }
    if (!header_done) {
        set_last_error("ply: %s has no end_header", path.c_str());
        return MLODS_ERR_INVALID;
    }
    const bool swap = fmt == PlyFormat::Be;
    for (const PlyElement& e : elems) {
        const bool is_vertex = e.name == "vertex";
        int ix[6] = {-1, -1, -1, -1, -1, -1};
        static const char* want[6] = {"x", "y", "z", "nx", "ny", "nz"};
        for (size_t k = 0; k < e.props.size(); ++k)
            for (int j = 0; j < 6; ++j)
                if (e.props[k].name == want[j] && !e.props[k].list) ix[j] = int(k);
        if (is_vertex && (ix[0] < 0 || ix[1] < 0 || ix[2] < 0)) {
            set_last_error("ply: the vertex element has no x, y, z");
            return MLODS_ERR_INVALID;
        }
        const bool normals = is_vertex && ix[3] >= 0 && ix[4] >= 0 && ix[5] >= 0;
        if (is_vertex) {
            c.pos.assign(size_t(e.count) * 3, 0.f);
            if (normals) c.nrm.assign(size_t(e.count) * 3, 0.f);
            c.has_normals = normals;
        }
        std::vector<double> vals(e.props.size());
        for (int64_t r = 0; r < e.count; ++r) {
            for (size_t k = 0; k < e.props.size(); ++k) {
                const PlyProp& p = e.props[k];
                if (fmt == PlyFormat::Ascii) {
                    double v = 0;
                    if (p.list) {
                        int64_t cnt = 0;
                        in >> cnt;
                        for (int64_t q = 0; q < cnt; ++q) in >> v;
                        v = 0;
                    } else {
                        in >> v;
                    }
                    if (!in) {
                        set_last_error("ply: truncated ascii data");
                        return MLODS_ERR_INVALID;
                    }
                    vals[k] = v;
                } else {
                    unsigned char b[8];
                    if (p.list) {
                        if (!in.read(reinterpret_cast<char*>(b), p.count_size)) {
                            set_last_error("ply: truncated binary data");
                            return MLODS_ERR_INVALID;
                        }
                        const int64_t cnt = int64_t(decode(b, p.count_size, p.count_kind, swap));
                        in.ignore(cnt * p.size);
                        vals[k] = 0;
                    } else {
                        if (!in.read(reinterpret_cast<char*>(b), p.size)) {
                            set_last_error("ply: truncated binary data");
                            return MLODS_ERR_INVALID;
                        }
                        vals[k] = decode(b, p.size, p.kind, swap);
                    }
                }
            }
            if (is_vertex) {
                for (int j = 0; j < 3; ++j) c.pos[3 * size_t(r) + size_t(j)] = float(vals[size_t(ix[j])]);
                if (normals)
                    for (int j = 0; j < 3; ++j) c.nrm[3 * size_t(r) + size_t(j)] = float(vals[size_t(ix[3 + j])]);
            }
        }
        if (is_vertex) return MLODS_OK;  // what follows (faces) is not needed
    }
    set_last_error("ply: %s has no vertex element", path.c_str());
    return MLODS_ERR_INVALID;
}

int read_pn(const std::string& path, mlods_cloud_s& c)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        set_last_error("pn: cannot open %s", path.c_str());
        return MLODS_ERR_INVALID;
    }
    std::vector<float> buf(6 * 4096);
    c.pos.clear();
    c.nrm.clear();
    for (;;) {
        const size_t got = std::fread(buf.data(), 4, buf.size(), f);
        for (size_t i = 0; i + 6 <= got; i += 6) {  // complete records, as Pn::load reads them
            c.pos.insert(c.pos.end(), &buf[i], &buf[i] + 3);
            c.nrm.insert(c.nrm.end(), &buf[i] + 3, &buf[i] + 6);
        }
        if (got < buf.size()) break;
    }
    std::fclose(f);
    c.has_normals = true;
    return MLODS_OK;
}

// Pn::normalize, Pn.cpp:262-290 (float arithmetic in the same order)
void normalize(mlods_cloud_s& c)
{
    const size_t n = c.pos.size() / 3;
    if (n == 0) return;
    float off[3], mx[3], mn[3];
    for (int a = 0; a < 3; ++a) off[a] = mx[a] = mn[a] = c.pos[size_t(a)];
    for (size_t i = 1; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            const float v = c.pos[3 * i + size_t(a)];
            off[a] += v;
            mx[a] = std::max(v, mx[a]);
            mn[a] = std::min(v, mn[a]);
        }
    for (int a = 0; a < 3; ++a) {
        off[a] /= float(n);
        mx[a] -= off[a];
        mn[a] -= off[a];
    }
    float d2 = 0.f;
    for (int a = 0; a < 3; ++a) d2 += (mx[a] - mn[a]) * (mx[a] - mn[a]);
    const float small = std::sqrt(d2) * 0.005f;
    for (int a = 0; a < 3; ++a) {
        mx[a] += small;
        mn[a] -= small;
    }
    float norme = std::fabs(mx[0]);
    const float cand[5] = {std::fabs(mx[1]), std::fabs(mx[2]), std::fabs(mn[0]), std::fabs(mn[1]), std::fabs(mn[2])};
    for (float v : cand) norme = std::max(norme, v);
    for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) c.pos[3 * i + size_t(a)] = (c.pos[3 * i + size_t(a)] - off[a]) / norme;
    for (int a = 0; a < 3; ++a) c.offset[a] = off[a];
    c.norme = norme;
}

template <typename T>
void put(std::vector<unsigned char>& out, const T& v)
{
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    out.insert(out.end(), p, p + sizeof(T));
}

template <typename T>
bool get(const unsigned char*& p, const unsigned char* end, T& v)
{
    if (size_t(end - p) < sizeof(T)) return false;
    std::memcpy(&v, p, sizeof(T));
    p += sizeof(T);
    return true;
}

}  // namespace
}  // namespace mlods

using namespace mlods;

extern "C" {

int mlods_cloud_load(const char* path, int32_t do_normalize, mlods_cloud* out)
{
    if (!path || !out) {
        set_last_error("cloud load: bad arguments");
        return MLODS_ERR_INVALID;
    }
    *out = nullptr;
    auto* c = new (std::nothrow) mlods_cloud_s();
    if (!c) {
        set_last_error("cloud load: host allocation failed");
        return MLODS_ERR_CAPACITY;
    }
    const std::string p(path);
    int rc;
    if (ends_with(p, "pn")) rc = read_pn(p, *c);
    else if (ends_with(p, "ply")) rc = read_ply(p, *c);
    else {
        set_last_error("cloud load: %s is neither .pn nor .ply", path);
        rc = MLODS_ERR_INVALID;
    }
    if (rc == MLODS_OK && do_normalize) normalize(*c);
    if (rc != MLODS_OK) {
        delete c;
        return rc;
    }
    *out = c;
    return MLODS_OK;
}

int mlods_cloud_info(mlods_cloud c, int64_t* n_points, int32_t* has_normals, float* offset, float* norme)
{
    if (!c) {
        set_last_error("null cloud");
        return MLODS_ERR_INVALID;
    }
    if (n_points) *n_points = int64_t(c->pos.size() / 3);
    if (has_normals) *has_normals = c->has_normals ? 1 : 0;
    if (offset) std::memcpy(offset, c->offset, sizeof c->offset);
    if (norme) *norme = c->norme;
    return MLODS_OK;
}

int mlods_cloud_get(mlods_cloud c, float* pts, float* nrm)
{
    if (!c) {
        set_last_error("null cloud");
        return MLODS_ERR_INVALID;
    }
    if (pts) std::memcpy(pts, c->pos.data(), c->pos.size() * sizeof(float));
    if (nrm && c->has_normals) std::memcpy(nrm, c->nrm.data(), c->nrm.size() * sizeof(float));
    return MLODS_OK;
}

int mlods_cloud_free(mlods_cloud c)
{
    delete c;
    return MLODS_OK;
}

int mlods_cloud_save(const char* path, const float* pts, const float* nrm, int64_t n, const float* offset,
                     float norme)
{
    if (!path || (!pts && n > 0) || n < 0) {
        set_last_error("cloud save: bad arguments");
        return MLODS_ERR_INVALID;
    }
    const float zero[3] = {0.f, 0.f, 0.f};
    const float* off = offset ? offset : zero;
    const std::string p(path);
    std::vector<unsigned char> body;
    body.reserve(size_t(n) * 24);
    for (int64_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) put(body, pts[3 * i + a] * norme + off[a]);  // realPosition
        if (nrm)
            for (int a = 0; a < 3; ++a) put(body, nrm[3 * i + a]);
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        set_last_error("cloud save: cannot write %s", path);
        return MLODS_ERR_INVALID;
    }
    bool ok = true;
    if (ends_with(p, "ply")) {
        std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n) +
                        "\nproperty float x\nproperty float y\nproperty float z\n";
        if (nrm) h += "property float nx\nproperty float ny\nproperty float nz\n";
        h += "end_header\n";
        ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
    } else if (!ends_with(p, "pn") || !nrm) {
        std::fclose(f);
        set_last_error("cloud save: %s needs a .ply name (or .pn with normals)", path);
        return MLODS_ERR_INVALID;
    }
    ok = ok && std::fwrite(body.data(), 1, body.size(), f) == body.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        set_last_error("cloud save: write to %s failed", path);
        return MLODS_ERR_INVALID;
    }
    return MLODS_OK;
}

int mlods_cloud_normalize(const float* pts, int64_t n, float* out_pts, float* offset, float* norme)
{
    if (!pts || !out_pts || n <= 0) {
        set_last_error("cloud normalize: bad arguments");
        return MLODS_ERR_INVALID;
    }
    mlods_cloud_s c;
    c.pos.assign(pts, pts + 3 * n);
    normalize(c);
    std::memcpy(out_pts, c.pos.data(), c.pos.size() * sizeof(float));
    if (offset) std::memcpy(offset, c.offset, sizeof c.offset);
    if (norme) *norme = c.norme;
    return MLODS_OK;
}

// Pn::order (Pn.cpp:388-440): Morton codes of the points on a grid^3 lattice
// over the cube [min, max]^3 of the box's extreme coordinates (x to bits
// 1, 4, 7..., y to 0, 3, 6..., z to 2, 5, 8...), points sorted by code.  The
// reference's std::sort leaves equal codes in unspecified order; here they
// keep their input order (counting sort).
int mlods_cloud_morton_order(const float* pts, int64_t n, int32_t grid, uint32_t* perm)
{
    if (!pts || !perm || n < 0 || n >= (int64_t(1) << 32) || grid < 1 || grid > 1024) {
        set_last_error("cloud morton order: bad arguments");
        return MLODS_ERR_INVALID;
    }
    if (n == 0) return MLODS_OK;
    float mn[3], mx[3];
    for (int a = 0; a < 3; ++a) mn[a] = mx[a] = pts[a];
    for (int64_t i = 1; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            const float v = pts[3 * i + a];
            if (v < mn[a]) mn[a] = v;
            if (v > mx[a]) mx[a] = v;
        }
    const float lo = std::min(std::min(mn[0], mn[1]), mn[2]);
    const float hi = std::max(std::max(mx[0], mx[1]), mx[2]);
    const float norme = hi - lo;
    int bits = 0;
    while ((1 << bits) < grid) ++bits;
    std::vector<uint32_t> code(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c[3];
        for (int a = 0; a < 3; ++a) {
            const float t = std::floor((pts[3 * i + a] - lo) / norme * float(grid));
            c[a] = (t > 0.f) ? std::min(uint32_t(t), uint32_t(grid - 1)) : 0u;  // glm::clamp to [0, grid-1]
        }
        uint32_t m = 0;
        for (int b = 0; b < bits && 3 * b + 2 < 32; ++b)
            m |= ((c[1] >> b) & 1u) << (3 * b) | ((c[0] >> b) & 1u) << (3 * b + 1) | ((c[2] >> b) & 1u) << (3 * b + 2);
        code[size_t(i)] = m;
    }
    const size_t ncodes = size_t(1) << std::min(30, 3 * bits);
    std::vector<uint32_t> start(ncodes + 1, 0);
    for (uint32_t m : code) ++start[m + 1];
    for (size_t k = 0; k < ncodes; ++k) start[k + 1] += start[k];
    for (int64_t i = 0; i < n; ++i) perm[start[code[size_t(i)]]++] = uint32_t(i);
    return MLODS_OK;
}

// Pn::initialize(n, pointSetToFit, factor) (Pn.cpp:324-357): n queries, each
// a random input point moved by a random vector of the disk of radius
// meanGap in its tangent plane (meanGap = 2 * cbrt(pi / n_points) * factor,
// Pn::computeMeanGap, Pn.cpp:170-176).  The reference draws from rand() and
// a std::random_device seed; here one seeded std::mt19937 does.
int mlods_cloud_sample_around(const float* pts, const float* nrm, int64_t n_pts, int64_t n_out, float factor,
                              uint64_t seed, float* out_pts, float* out_nrm)
{
    if (!pts || !nrm || n_pts <= 0 || n_out < 0 || !out_pts) {
        set_last_error("cloud sample: bad arguments");
        return MLODS_ERR_INVALID;
    }
    const float r = 0.5f;
    const float surface = 4.f * float(M_PI) * r * r;
    const float gap = (std::cbrt(surface / float(n_pts)) * 2.f) * factor;
    std::mt19937_64 mt(seed);
    std::uniform_int_distribution<int64_t> pick(0, n_pts - 1);
    std::uniform_real_distribution<float> unit(0.f, 1.f);
    auto cross = [](const float* a, const float* b, float* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    auto normalize3 = [](float* v) {
        const float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int a = 0; a < 3; ++a) v[a] /= l;
    };
    for (int64_t i = 0; i < n_out; ++i) {
        const int64_t k = pick(mt);
        const float* p = pts + 3 * k;
        const float* nv = nrm + 3 * k;
        static const float ez[3] = {0.f, 0.f, 1.f}, ey[3] = {0.f, 1.f, 0.f};
        float e1[3], e2[3];
        cross(nv, nv[2] != 0.f ? ez : ey, e1);  // dot(n, (0, 0, 1)) != 0
        normalize3(e1);
        cross(nv, e1, e2);
        normalize3(e2);
        const float rr = gap * std::sqrt(unit(mt));
        const float th = unit(mt) * 2.f * float(M_PI);
        for (int a = 0; a < 3; ++a) out_pts[3 * i + a] = p[a] + (rr * std::cos(th) * e1[a] + rr * std::sin(th) * e2[a]);
        if (out_nrm)
            for (int a = 0; a < 3; ++a) out_nrm[3 * i + a] = nv[a];
    }
    return MLODS_OK;
}

// scene::loadParameters, scene.cpp:1183-1250: packed fields in this order
int mlods_params_file_load(const char* path, mlods_scene_params* p)
{
    if (!path || !p) {
        set_last_error("params load: bad arguments");
        return MLODS_ERR_INVALID;
    }
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        set_last_error("params load: cannot open %s", path);
        return MLODS_ERR_INVALID;
    }
    std::vector<unsigned char> b((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    const unsigned char* q = b.data();
    const unsigned char* end = q + b.size();
    std::memset(p, 0, sizeof *p);
    bool ok = true;
    for (float& v : p->cam_quat) ok = ok && get(q, end, v);
    for (float& v : p->cam_translation) ok = ok && get(q, end, v);
    ok = ok && get(q, end, p->cam_dist) && get(q, end, p->sigma);
    for (float& v : p->fixed_sigmas) ok = ok && get(q, end, v);
    ok = ok && get(q, end, p->beginning_sigma) && get(q, end, p->factor) && get(q, end, p->constant_shift) &&
         get(q, end, p->exponent) && get(q, end, p->cutoff) && get(q, end, p->n_computed_sigmas) &&
         get(q, end, p->max_iterations) && get(q, end, p->max_depth) && get(q, end, p->min_depth) &&
         get(q, end, p->fast_method) && get(q, end, p->kernel_type) && get(q, end, p->computed_sigma) &&
         get(q, end, p->cut) && get(q, end, p->n_points) && get(q, end, p->max_upsamples);
    for (float& v : p->offset) ok = ok && get(q, end, v);
    if (!ok) {
        set_last_error("params load: %s is shorter than the %d-byte layout", path, MLODS_PARAMS_FILE_BYTES);
        return MLODS_ERR_INVALID;
    }
    return MLODS_OK;
}

int mlods_params_file_save(const char* path, const mlods_scene_params* p)
{
    if (!path || !p) {
        set_last_error("params save: bad arguments");
        return MLODS_ERR_INVALID;
    }
    std::vector<unsigned char> b;
    for (float v : p->cam_quat) put(b, v);
    for (float v : p->cam_translation) put(b, v);
    put(b, p->cam_dist);
    put(b, p->sigma);
    for (float v : p->fixed_sigmas) put(b, v);
    put(b, p->beginning_sigma);
    put(b, p->factor);
    put(b, p->constant_shift);
    put(b, p->exponent);
    put(b, p->cutoff);
    put(b, p->n_computed_sigmas);
    put(b, p->max_iterations);
    put(b, p->max_depth);
    put(b, p->min_depth);
    put(b, p->fast_method);
    put(b, p->kernel_type);
    put(b, p->computed_sigma);
    put(b, p->cut);
    put(b, p->n_points);
    put(b, p->max_upsamples);
    for (float v : p->offset) put(b, v);
    std::ofstream out(path, std::ios::binary);
    if (!out || !out.write(reinterpret_cast<const char*>(b.data()), std::streamsize(b.size()))) {
        set_last_error("params save: cannot write %s", path);
        return MLODS_ERR_INVALID;
    }
    return MLODS_OK;
}

}  // extern "C"
