// fm_checkpoint.cpp — restart files in the byte layout of the reference's
// CheckpointFile (FEM/adaptive_fem_engine.hpp:1347-1452), so that states
// saved here and the reference's own restart files interchange:
//
//   u32 load_step, u32 adapt_iter, u32 n_nodes, u32 n_elements, u32 n_dofs
//   per node      6 x f64  x, y, z, u, v, w            (MeshNode)
//   per element   4 x u32 nodes, f64 volume, f64 jacobian_det,
//                 f64 quality_metric                    (TetraElement)
//   per element   9 x f64 F, 6 x f64 stress, 6 x f64 eps_plastic,
//                 f64 kappa, f64 gamma_p                 (ElementState)
//   n_dofs x f64  solution
//
// little-endian, no padding.  The reference writes field by field; here
// each section is packed into a buffer and written (or read) in one call.
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "fm_api.h"

namespace {

constexpr size_t kNodeBytes = 6 * 8;
constexpr size_t kElemBytes = 4 * 4 + 3 * 8;
constexpr size_t kStateBytes = 23 * 8;

template <typename T>
void put(unsigned char*& p, T v) {
    std::memcpy(p, &v, sizeof v);
    p += sizeof v;
}
template <typename T>
T get(const unsigned char*& p) {
    T v;
    std::memcpy(&v, p, sizeof v);
    p += sizeof v;
    return v;
}

struct File {
    FILE* f = nullptr;
    File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace

extern "C" {

fm_status fm_checkpoint_save(const char* path, const fm_checkpoint* ck) {
    if (!path || !ck || !ck->xyz || !ck->conn || (ck->n_dofs && !ck->u)) return FM_ERR_ARG;
    try {
        File out(path, "wb");
        if (!out.f) return FM_ERR_ARG;
        const uint32_t nn = ck->n_nodes, ne = ck->n_elems;
        std::vector<unsigned char> buf(20 + (size_t)nn * kNodeBytes);
        unsigned char* p = buf.data();
        put(p, ck->load_step);
        put(p, ck->adapt_iter);
        put(p, nn);
        put(p, ne);
        put(p, ck->n_dofs);
        for (size_t n = 0; n < nn; ++n) {
            for (int d = 0; d < 3; ++d) put(p, ck->xyz[3 * n + d]);
            for (int d = 0; d < 3; ++d) put(p, ck->node_disp ? ck->node_disp[3 * n + d] : 0.0);
        }
        if (std::fwrite(buf.data(), 1, buf.size(), out.f) != buf.size()) return FM_ERR_ARG;
        buf.assign((size_t)ne * kElemBytes, 0);
        p = buf.data();
        for (size_t e = 0; e < ne; ++e) {
            for (int v = 0; v < 4; ++v) put(p, ck->conn[4 * e + v]);
            put(p, ck->volume ? ck->volume[e] : 0.0);
            put(p, ck->jacobian_det ? ck->jacobian_det[e] : 0.0);
            put(p, ck->quality ? ck->quality[e] : 0.0);
        }
        if (std::fwrite(buf.data(), 1, buf.size(), out.f) != buf.size()) return FM_ERR_ARG;
        buf.assign((size_t)ne * kStateBytes, 0);
        p = buf.data();
        for (size_t e = 0; e < ne; ++e) {
            // ElementState::initialize values where the caller has none
            for (int i = 0; i < 9; ++i) put(p, ck->F ? ck->F[9 * e + i] : (i % 4 == 0 ? 1.0 : 0.0));
            for (int i = 0; i < 6; ++i) put(p, ck->stress ? ck->stress[6 * e + i] : 0.0);
            for (int i = 0; i < 6; ++i) put(p, ck->eps_plastic ? ck->eps_plastic[6 * e + i] : 0.0);
            put(p, ck->kappa ? ck->kappa[e] : 0.0);
            put(p, ck->gamma_p ? ck->gamma_p[e] : 0.0);
        }
        if (std::fwrite(buf.data(), 1, buf.size(), out.f) != buf.size()) return FM_ERR_ARG;
        if (ck->n_dofs &&
            std::fwrite(ck->u, sizeof(double), ck->n_dofs, out.f) != (size_t)ck->n_dofs)
            return FM_ERR_ARG;
    } catch (const std::bad_alloc&) {
        return FM_ERR_OOM;
    }
    return FM_OK;
}

fm_status fm_checkpoint_header(const char* path, fm_checkpoint* ck) {
    if (!path || !ck) return FM_ERR_ARG;
    File in(path, "rb");
    if (!in.f) return FM_ERR_ARG;
    unsigned char h[20];
    if (std::fread(h, 1, 20, in.f) != 20) return FM_ERR_ARG;
    const unsigned char* p = h;
    ck->load_step = get<uint32_t>(p);
    ck->adapt_iter = get<uint32_t>(p);
    ck->n_nodes = get<uint32_t>(p);
    ck->n_elems = get<uint32_t>(p);
    ck->n_dofs = get<uint32_t>(p);
    return FM_OK;
}

fm_status fm_checkpoint_load(const char* path, fm_checkpoint* ck) {
    if (!path || !ck) return FM_ERR_ARG;
    fm_checkpoint h;
    std::memset(&h, 0, sizeof h);
    fm_status st = fm_checkpoint_header(path, &h);
    if (st != FM_OK) return st;
    if (h.n_nodes != ck->n_nodes || h.n_elems != ck->n_elems || h.n_dofs != ck->n_dofs)
        return FM_ERR_ARG;  // the caller sizes its arrays from fm_checkpoint_header
    try {
        File in(path, "rb");
        if (!in.f || std::fseek(in.f, 20, SEEK_SET) != 0) return FM_ERR_ARG;
        ck->load_step = h.load_step;
        ck->adapt_iter = h.adapt_iter;
        const uint32_t nn = h.n_nodes, ne = h.n_elems;
        std::vector<unsigned char> buf((size_t)nn * kNodeBytes);
        if (std::fread(buf.data(), 1, buf.size(), in.f) != buf.size()) return FM_ERR_ARG;
        const unsigned char* p = buf.data();
        for (size_t n = 0; n < nn; ++n) {
            for (int d = 0; d < 3; ++d) {
                const double v = get<double>(p);
                if (ck->xyz) ck->xyz[3 * n + d] = v;
            }
            for (int d = 0; d < 3; ++d) {
                const double v = get<double>(p);
                if (ck->node_disp) ck->node_disp[3 * n + d] = v;
            }
        }
        buf.resize((size_t)ne * kElemBytes);
        if (std::fread(buf.data(), 1, buf.size(), in.f) != buf.size()) return FM_ERR_ARG;
        p = buf.data();
        for (size_t e = 0; e < ne; ++e) {
            for (int v = 0; v < 4; ++v) {
                const uint32_t id = get<uint32_t>(p);
                if (ck->conn) ck->conn[4 * e + v] = id;
            }
            const double vol = get<double>(p), jd = get<double>(p), q = get<double>(p);
            if (ck->volume) ck->volume[e] = vol;
            if (ck->jacobian_det) ck->jacobian_det[e] = jd;
            if (ck->quality) ck->quality[e] = q;
        }
        buf.resize((size_t)ne * kStateBytes);
        if (std::fread(buf.data(), 1, buf.size(), in.f) != buf.size()) return FM_ERR_ARG;
        p = buf.data();
        for (size_t e = 0; e < ne; ++e) {
            for (int i = 0; i < 9; ++i) {
                const double v = get<double>(p);
                if (ck->F) ck->F[9 * e + i] = v;
            }
            for (int i = 0; i < 6; ++i) {
                const double v = get<double>(p);
                if (ck->stress) ck->stress[6 * e + i] = v;
            }
            for (int i = 0; i < 6; ++i) {
                const double v = get<double>(p);
                if (ck->eps_plastic) ck->eps_plastic[6 * e + i] = v;
            }
            const double k = get<double>(p), g = get<double>(p);
            if (ck->kappa) ck->kappa[e] = k;
            if (ck->gamma_p) ck->gamma_p[e] = g;
        }
        if (h.n_dofs) {
            std::vector<double> u(h.n_dofs);
            if (std::fread(u.data(), sizeof(double), h.n_dofs, in.f) != (size_t)h.n_dofs)
                return FM_ERR_ARG;
            if (ck->u) std::memcpy(ck->u, u.data(), sizeof(double) * h.n_dofs);
        }
    } catch (const std::bad_alloc&) {
        return FM_ERR_OOM;
    }
    return FM_OK;
}

}  // extern "C"
