// XDMF output that doubles as a checkpoint, in the file format of the reference's XDMFOutput
// (src/terra/io/xdmf.hpp:13-148 format description, :293-512 write(), :578-650 mesh, :656-900 attributes,
// :898-1060 metadata), so that its checkpoint reader and Paraview read what this library writes.
//
// A writer is bound to one level of a shell (one subdomain per diamond). Fields are registered once (scalar or
// 3-vector, FP64 or FP32 device data, written as 4- or 8-byte floats) and every write() copies them to the host
// and writes `<name>_<step>.bin` per field and `step_<step>.xmf`; the first write() also writes geometry.bin
// (physical node coordinates), topology.bin (two wedges per hex cell, int64), checkpoint_metadata.bin and a
// README. Binary order per diamond: r, then y, then x fastest, then the vector component. tn_xdmf_read restores a
// field from such a directory into device memory.
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/terra_b200.h"
#include "tn_runtime.hpp"

namespace tn {
namespace {

struct Field {
    std::string        name;
    int                precision = 0;  // device data: 0 f64, 1 f32
    int                ncomp     = 1;
    std::vector<void*> comps;
    int                out_bytes = 4;
};

std::string xml_escape(const std::string& s)
{
    std::string o;
    for (char c : s) {
        switch (c) {
        case '&': o += "&amp;"; break;
        case '"': o += "&quot;"; break;
        case '\'': o += "&apos;"; break;
        case '<': o += "&lt;"; break;
        case '>': o += "&gt;"; break;
        default: o += c;
        }
    }
    return o;
}

void write_file(const std::string& path, const std::string& bytes)
{
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) throw Error(kErrArg, "cannot open " + path + " for writing");
    f.write(bytes.data(), static_cast<std::streamsize>(bytes.size()));
    if (!f) throw Error(kErrArg, "write to " + path + " failed");
}

template <typename T>
void put(std::string& out, T v)
{
    out.append(reinterpret_cast<const char*>(&v), sizeof(T));
}

void ensure_directory(const std::string& dir)
{
    std::string partial;
    for (size_t i = 0; i <= dir.size(); ++i) {
        if (i == dir.size() || dir[i] == '/') {
            if (!partial.empty() && mkdir(partial.c_str(), 0755) != 0 && errno != EEXIST)
                throw Error(kErrArg, "cannot create directory " + partial);
        }
        if (i < dir.size()) partial += dir[i];
    }
}

// host copy of ncomp components (each nodes() values) as doubles
std::vector<double> fetch(const DeviceLevel& L, const Field& f)
{
    const int64_t       n = L.nodes();
    std::vector<double> h(static_cast<size_t>(n) * f.ncomp);
    for (int c = 0; c < f.ncomp; ++c) {
        if (f.precision == 0) {
            cuda_check(cudaMemcpy(h.data() + c * n, f.comps[c], sizeof(double) * n, cudaMemcpyDeviceToHost), "copy");
        } else {
            std::vector<float> t(static_cast<size_t>(n));
            cuda_check(cudaMemcpy(t.data(), f.comps[c], sizeof(float) * n, cudaMemcpyDeviceToHost), "copy");
            for (int64_t i = 0; i < n; ++i) h[c * n + i] = t[i];
        }
    }
    return h;
}

}  // namespace

struct Xdmf {
    const Shell*       shell = nullptr;
    int                level = 0;
    std::string        dir;
    int                geometry_bytes = 4;
    std::vector<Field> fields;
    int                step  = 0;
    bool               wrote = false;

    const DeviceLevel& lvl() const { return shell->level(level); }

    std::string mesh_geometry() const
    {
        const DeviceLevel& L = lvl();
        const int          nl = L.nl(), nr = L.nr();
        std::string        out;
        for (int d = 0; d < 10; ++d)
            for (int r = 0; r < nr; ++r)
                for (int y = 0; y < nl; ++y)
                    for (int x = 0; x < nl; ++x)
                        for (int k = 0; k < 3; ++k) {
                            const double v = L.host.coords[(static_cast<size_t>(d * nl + x) * nl + y) * 3 + k] *
                                             L.host.radii[r];
                            if (geometry_bytes == 4)
                                put<float>(out, static_cast<float>(v));
                            else
                                put<double>(out, v);
                        }
        return out;
    }

    std::string mesh_topology() const
    {
        const DeviceLevel& L  = lvl();
        const int64_t      nx = L.nl(), ny = L.nl(), nr = L.nr();
        std::string        out;
        for (int64_t d = 0; d < 10; ++d)
            for (int64_t r = 0; r < nr - 1; ++r)
                for (int64_t y = 0; y < ny - 1; ++y)
                    for (int64_t x = 0; x < nx - 1; ++x) {
                        const int64_t b = d * nx * ny * nr, v0 = b + r * nx * ny + y * nx + x, v4 = v0 + nx * ny;
                        const int64_t w0[6] = {v0, v0 + 1, v0 + nx, v4, v4 + 1, v4 + nx};
                        const int64_t w1[6] = {v0 + nx + 1, v0 + nx, v0 + 1, v4 + nx + 1, v4 + nx, v4 + 1};
                        for (int64_t v : w0) put<int64_t>(out, v);
                        for (int64_t v : w1) put<int64_t>(out, v);
                    }
        return out;
    }

    std::string field_data(const Field& f) const
    {
        const DeviceLevel&        L  = lvl();
        const int                 nl = L.nl(), nr = L.nr();
        const int64_t             n  = L.nodes();
        const std::vector<double> h  = fetch(L, f);
        std::string               out;
        out.reserve(static_cast<size_t>(n) * f.ncomp * f.out_bytes);
        for (int d = 0; d < 10; ++d)
            for (int r = 0; r < nr; ++r)
                for (int y = 0; y < nl; ++y)
                    for (int x = 0; x < nl; ++x) {
                        const int64_t i = (static_cast<int64_t>(d * nl + x) * nl + y) * nr + r;
                        for (int c = 0; c < f.ncomp; ++c) {
                            if (f.out_bytes == 4)
                                put<float>(out, static_cast<float>(h[c * n + i]));
                            else
                                put<double>(out, h[c * n + i]);
                        }
                    }
        return out;
    }

    std::string metadata() const
    {
        const DeviceLevel& L = lvl();
        std::string        out;
        put<int32_t>(out, 1);  // version
        put<int32_t>(out, 1);  // subdomains per diamond side (one subdomain per diamond)
        put<int32_t>(out, 1);  // subdomains in the radial direction
        put<int32_t>(out, L.nl());
        put<int32_t>(out, L.nl());
        put<int32_t>(out, L.nr());
        for (double r : L.host.radii) put<double>(out, r);
        put<int32_t>(out, geometry_bytes);
        // fields in the order the reference lists them: scalar FP32, scalar FP64, vector FP32, vector FP64 data
        std::vector<const Field*> order;
        for (int vec = 0; vec < 2; ++vec)
            for (int prec = 1; prec >= 0; --prec)
                for (const Field& f : fields)
                    if ((f.ncomp > 1) == (vec == 1) && f.precision == prec) order.push_back(&f);
        put<int32_t>(out, static_cast<int32_t>(order.size()));
        for (const Field* f : order) {
            put<int32_t>(out, static_cast<int32_t>(f->name.size()));
            out += f->name;
            put<int32_t>(out, 2);  // floating point
            put<int32_t>(out, f->out_bytes);
            put<int32_t>(out, f->ncomp);
        }
        put<int32_t>(out, 0);  // subdomain ordering: explicit list of global subdomain ids
        for (int64_t d = 0; d < 10; ++d) put<int64_t>(out, d << 57);
        return out;
    }

    void write()
    {
        const DeviceLevel& L      = lvl();
        const int64_t      nodes  = L.nodes();
        const int64_t      elems  = 20ll * (L.nl() - 1) * (L.nl() - 1) * (L.nr() - 1);
        if (!wrote) {
            ensure_directory(dir);
            write_file(dir + "/README.md",
                       "XDMF output of a spherical-shell level (terra_b200): open step_*.xmf in an XDMF reader.\n"
                       "geometry.bin holds the node coordinates, topology.bin the wedge connectivity,\n"
                       "checkpoint_metadata.bin what a checkpoint reader needs, <field>_<step>.bin the values.\n");
            write_file(dir + "/geometry.bin", mesh_geometry());
            write_file(dir + "/topology.bin", mesh_topology());
            write_file(dir + "/checkpoint_metadata.bin", metadata());
        }
        std::ostringstream x;
        x << "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n";
        x << "<Xdmf Version=\"2.0\">\n  <Domain>\n    <Grid GridType=\"Uniform\" Name=\"Grid\">\n";
        x << "      <Geometry Type=\"XYZ\">\n        <DataItem DataType=\"Float\" Dimensions=\"" << nodes
          << " 3\" Endian=\"Little\" Format=\"Binary\" Precision=\"" << geometry_bytes
          << "\">geometry.bin</DataItem>\n      </Geometry>\n";
        x << "      <Topology NumberOfElements=\"" << elems << "\" Type=\"Wedge\">\n        <DataItem DataType=\"Int\" "
          << "Dimensions=\"" << elems * 6
          << "\" Endian=\"Little\" Format=\"Binary\" Precision=\"8\">topology.bin</DataItem>\n      </Topology>\n";
        for (const Field& f : fields) {
            const std::string file = f.name + "_" + std::to_string(step) + ".bin";
            write_file(dir + "/" + file, field_data(f));
            x << "      <Attribute AttributeType=\"" << (f.ncomp > 1 ? "Vector" : "Scalar") << "\" Center=\"Node\" Name=\""
              << xml_escape(f.name) << "\">\n        <DataItem DataType=\"Float\" Dimensions=\"" << nodes;
            if (f.ncomp > 1) x << " " << f.ncomp;
            x << "\" Endian=\"Little\" Format=\"Binary\" Precision=\"" << f.out_bytes << "\">" << xml_escape(file)
              << "</DataItem>\n      </Attribute>\n";
        }
        x << "    </Grid>\n  </Domain>\n</Xdmf>\n";
        write_file(dir + "/step_" + std::to_string(step) + ".xmf", x.str());
        ++step;
        wrote = true;
    }
};

// read_xdmf_checkpoint_grid: a field written by a writer of the same level layout
void xdmf_read(const Shell* sh, int level, const std::string& dir, const std::string& name, int step, int precision,
               int ncomp, void* const* comps)
{
    const DeviceLevel& L = sh->level(level);
    std::ifstream      m(dir + "/checkpoint_metadata.bin", std::ios::binary);
    if (!m) throw Error(kErrArg, "no checkpoint metadata in " + dir);
    auto get32 = [&]() {
        int32_t v = 0;
        m.read(reinterpret_cast<char*>(&v), sizeof(v));
        if (!m) throw Error(kErrArg, "truncated checkpoint metadata");
        return v;
    };
    if (get32() != 1) throw Error(kErrUnsupported, "unknown checkpoint version");
    const int32_t sd_lat = get32(), sd_rad = get32(), sx = get32(), sy = get32(), sr = get32();
    if (sd_lat != 1 || sd_rad != 1 || sx != L.nl() || sy != L.nl() || sr != L.nr())
        throw Error(kErrArg, "checkpoint layout does not match the level");
    m.seekg(static_cast<std::streamoff>(sizeof(double)) * sr, std::ios::cur);
    (void) get32();  // geometry bytes
    const int32_t nfiles = get32();
    int           bytes = 0, vdim = 0;
    for (int i = 0; i < nfiles; ++i) {
        const int32_t len = get32();
        std::string   s(static_cast<size_t>(len), '\0');
        m.read(s.data(), len);
        (void) get32();
        const int32_t b = get32(), v = get32();
        if (s == name) bytes = b, vdim = v;
    }
    if (bytes == 0) throw Error(kErrArg, "field " + name + " is not in the checkpoint");
    if (vdim != ncomp) throw Error(kErrArg, "component count differs from the checkpoint's");
    if (get32() != 0) throw Error(kErrUnsupported, "unknown subdomain ordering");
    std::vector<int64_t> ids(10);
    for (auto& id : ids) {
        m.read(reinterpret_cast<char*>(&id), sizeof(id));
        if (!m) throw Error(kErrArg, "truncated checkpoint metadata");
    }
    std::ifstream f(dir + "/" + name + "_" + std::to_string(step) + ".bin", std::ios::binary);
    if (!f) throw Error(kErrArg, "no data file for " + name + " step " + std::to_string(step));
    const int nl = L.nl(), nr = L.nr();
    const int64_t n = L.nodes();
    std::vector<double> h(static_cast<size_t>(n) * ncomp);
    for (int slot = 0; slot < 10; ++slot) {
        const int d = static_cast<int>(ids[slot] >> 57);
        if (d < 0 || d >= 10 || (ids[slot] & ((int64_t(1) << 57) - 1)) != 0)
            throw Error(kErrArg, "unexpected subdomain id in the checkpoint");
        for (int r = 0; r < nr; ++r)
            for (int y = 0; y < nl; ++y)
                for (int x = 0; x < nl; ++x)
                    for (int c = 0; c < ncomp; ++c) {
                        double v;
                        if (bytes == 4) {
                            float t;
                            f.read(reinterpret_cast<char*>(&t), 4);
                            v = t;
                        } else {
                            f.read(reinterpret_cast<char*>(&v), 8);
                        }
                        h[c * n + (static_cast<int64_t>(d * nl + x) * nl + y) * nr + r] = v;
                    }
    }
    if (!f) throw Error(kErrArg, "truncated data file");
    for (int c = 0; c < ncomp; ++c) {
        if (precision == 0) {
            cuda_check(cudaMemcpy(comps[c], h.data() + c * n, sizeof(double) * n, cudaMemcpyHostToDevice), "copy");
        } else {
            std::vector<float> t(h.begin() + c * n, h.begin() + (c + 1) * n);
            cuda_check(cudaMemcpy(comps[c], t.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "copy");
        }
    }
}

}  // namespace tn

namespace tn {

Xdmf* xdmf_create(const Shell* sh, int level, const std::string& dir, int geometry_bytes)
{
    if (geometry_bytes != 4 && geometry_bytes != 8) throw Error(kErrArg, "geometry_bytes must be 4 or 8");
    sh->level(level);
    auto* x           = new Xdmf;
    x->shell          = sh;
    x->level          = level;
    x->dir            = dir;
    x->geometry_bytes = geometry_bytes;
    return x;
}

void xdmf_add(Xdmf* x, const std::string& name, int precision, int ncomp, void* const* comps, int out_bytes)
{
    if (x->wrote) throw Error(kErrState, "fields must be added before the first write");
    if (precision != 0 && precision != 1) throw Error(kErrArg, "bad precision");
    if (ncomp != 1 && ncomp != 3) throw Error(kErrArg, "ncomp must be 1 or 3");
    if (out_bytes != 4 && out_bytes != 8) throw Error(kErrArg, "output bytes must be 4 or 8");
    if (name.empty()) throw Error(kErrArg, "empty field name");
    for (const auto& f : x->fields)
        if (f.name == name) throw Error(kErrArg, "field names must be unique");
    Field f;
    f.name      = name;
    f.precision = precision;
    f.ncomp     = ncomp;
    f.comps.assign(comps, comps + ncomp);
    f.out_bytes = out_bytes;
    x->fields.push_back(f);
}

void xdmf_write(Xdmf* x) { x->write(); }
void xdmf_destroy(Xdmf* x) { delete x; }

}  // namespace tn
