/*
 * xr_compat.hpp — the reference's C++ call surface, header-only, over libxr.
 *
 * Code written against ixactly/Xray-directional-reconstruction's headers
 * (reconstruct/include/{reconstruct.cuh, geometry.h, volume.h, params.h},
 * direction/include/pca.cuh) compiles against this header instead and links
 * with libxr.so: same names, same argument meaning, same layouts.
 *
 * Differences, all deliberate:
 *   - init_params(tag) reads the settings file named by the XR_SETTINGS
 *     environment variable (or the optional second argument); the reference
 *     hard-codes its author's path (params.cu:43).
 *   - Volume's copy constructor / assignment allocate (the reference's memcpy
 *     into unallocated storage, volume.h:34-46).
 *   - Failures throw xr::Error (the reference prints and continues).
 *   - calcEigenVector(ct, md, evalue, x, y, z) computes one voxel on the host
 *     in FP64; calcEigenVectorAll does every voxel on the GPU.
 */
#ifndef XR_COMPAT_HPP
#define XR_COMPAT_HPP

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "xr.h"

namespace xr {
struct Error : std::runtime_error {
    xr_status status;
    Error(xr_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};
inline xr_ctx *&context() {
    static xr_ctx *c = nullptr;
    return c;
}
inline void check(xr_status s, const char *what) {
    if (s != XR_OK) {
        const char *m = context() ? xr_last_error(context()) : "";
        throw Error(s, std::string(what) + ": " + m);
    }
}
}  // namespace xr

/* ---- params.h:9-37 globals, filled by init_params ---- */
inline std::string PROJ_PATH;
inline std::string VOLUME_PATH;
inline std::string DIRECTION_PATH;
inline int BLOCK_SIZE = 32;
inline int NUM_BASIS_VECTOR = 0;
inline int NUM_PROJ_COND = 0;
inline float SRC_OBJ_DISTANCE = 0;
inline float SRC_DETECT_DISTANCE = 0;
inline int NUM_PROJ = 0;
inline int NUM_DETECT_U = 0;
inline int NUM_DETECT_V = 0;
inline float DETECTOR_SIZE = 0;
inline int NUM_VOXEL = 0;
inline int LOAD_INDEX[100];
inline float basisVector[3 * 32];

/* init_params, params.cu:42-104. */
inline void init_params(const std::string &tag, const std::string &json_path = "") {
    std::string path = json_path;
    if (path.empty()) {
        const char *e = std::getenv("XR_SETTINGS");
        if (!e) throw xr::Error(XR_ERR_ARG, "init_params: set XR_SETTINGS to the settings.json path");
        path = e;
    }
    if (xr::context()) {
        xr_destroy(xr::context());
        xr::context() = nullptr;
    }
    xr_ctx *c = nullptr;
    const xr_status s = xr_init_params(path.c_str(), tag.c_str(), 0, &c);
    if (s != XR_OK) throw xr::Error(s, "init_params(" + tag + ") from " + path);
    xr::context() = c;
    xr_scan sc;
    xr::check(xr_get_scan(c, &sc), "xr_get_scan");
    const char *pp, *vp, *dp;
    xr::check(xr_get_paths(c, &pp, &vp, &dp, LOAD_INDEX), "xr_get_paths");
    PROJ_PATH = pp;
    VOLUME_PATH = vp;
    DIRECTION_PATH = dp;
    NUM_BASIS_VECTOR = sc.num_basis;
    NUM_PROJ_COND = sc.num_cond;
    SRC_OBJ_DISTANCE = sc.sod;
    SRC_DETECT_DISTANCE = sc.sdd;
    NUM_PROJ = sc.num_proj;
    NUM_DETECT_U = NUM_DETECT_V = sc.num_detect;
    DETECTOR_SIZE = sc.det_size;
    NUM_VOXEL = sc.num_voxel;
    for (int i = 0; i < 3 * sc.num_basis; i++) basisVector[i] = sc.basis[i];
}

/* geometry.h:8-25 */
class Geometry {
  public:
    Geometry(float sdd, float sod, float detSize, int voxel, int detect, int nProj)
        : sdd(sdd), sod(sod), detSize(detSize), voxel(voxel), detect(detect), nProj(nProj) {
        voxSize = sod * detSize / sdd;
    }
    float sdd;
    float sod;
    float voxSize;
    float detSize;
    int voxel;
    int detect;
    int nProj;
};

/* volume.h:18-165: host 3-D array, x fastest. */
template <typename T>
class Volume {
  public:
    Volume() : sizeX(0), sizeY(0), sizeZ(0) {}
    explicit Volume(int64_t x, int64_t y, int64_t z) : sizeX(x), sizeY(y), sizeZ(z) {
        data = std::make_unique<T[]>(x * y * z);
    }
    explicit Volume(std::string &filename, int64_t x, int64_t y, int64_t z) { load(filename, x, y, z); }
    Volume(const Volume &v) : sizeX(v.sizeX), sizeY(v.sizeY), sizeZ(v.sizeZ) {
        data = std::make_unique<T[]>(sizeX * sizeY * sizeZ);
        if (v.data) std::memcpy(data.get(), v.data.get(), sizeof(T) * sizeX * sizeY * sizeZ);
    }
    Volume &operator=(const Volume &v) {
        if (this == &v) return *this;
        sizeX = v.sizeX, sizeY = v.sizeY, sizeZ = v.sizeZ;
        data = std::make_unique<T[]>(sizeX * sizeY * sizeZ);
        if (v.data) std::memcpy(data.get(), v.data.get(), sizeof(T) * sizeX * sizeY * sizeZ);
        return *this;
    }
    Volume(Volume &&v) noexcept : sizeX(v.sizeX), sizeY(v.sizeY), sizeZ(v.sizeZ), data(std::move(v.data)) {
        v.sizeX = v.sizeY = v.sizeZ = 0;
    }
    Volume &operator=(Volume &&v) noexcept {
        sizeX = v.sizeX, sizeY = v.sizeY, sizeZ = v.sizeZ;
        v.sizeX = v.sizeY = v.sizeZ = 0;
        data = std::move(v.data);
        return *this;
    }
    T &operator()(int64_t x, int64_t y, int64_t z) { return data[z * (sizeX * sizeY) + y * sizeX + x]; }
    T operator()(int64_t x, int64_t y, int64_t z) const { return data[z * (sizeX * sizeY) + y * sizeX + x]; }
    T *get() const { return data.get(); }
    T mean() const {
        double m = 0;
        const int64_t n = sizeX * sizeY * sizeZ;
        for (int64_t i = 0; i < n; i++) m += data[i] / static_cast<double>(n);
        return static_cast<T>(m);
    }
    void set(int64_t x, int64_t y, int64_t z) {
        sizeX = x, sizeY = y, sizeZ = z;
        data = std::make_unique<T[]>(x * y * z);
    }
    void load(const std::string &filename, int64_t x, int64_t y, int64_t z) {
        set(x, y, z);
        std::ifstream f(filename, std::ios::binary);
        if (!f) throw xr::Error(XR_ERR_IO, "Volume::load: cannot open " + filename);
        f.read(reinterpret_cast<char *>(data.get()), sizeof(T) * x * y * z);
        if (f.gcount() != (std::streamsize)(sizeof(T) * x * y * z))
            throw xr::Error(XR_ERR_IO, "Volume::load: short file " + filename);
    }
    void save(const std::string &filename) const {
        std::ofstream f(filename, std::ios::binary);
        if (!f) throw xr::Error(XR_ERR_IO, "Volume::save: cannot open " + filename);
        f.write(reinterpret_cast<const char *>(data.get()), sizeof(T) * sizeX * sizeY * sizeZ);
    }
    void forEach(const std::function<T(T)> &f) {
        const int64_t n = sizeX * sizeY * sizeZ;
        for (int64_t i = 0; i < n; i++) data[i] = f(data[i]);
    }
    int64_t x() const { return sizeX; }
    int64_t y() const { return sizeY; }
    int64_t z() const { return sizeZ; }

  private:
    int64_t sizeX, sizeY, sizeZ;
    std::unique_ptr<T[]> data;
};

/* reconstruct.cuh:14-24 */
enum class Method { XTT, MLEM, ART, FDK };
enum class Rotate { CW, CCW };

namespace xr {
inline xr_ctx *need() {
    if (!context()) throw Error(XR_ERR_STATE, "call init_params(tag) first");
    return context();
}
inline xr_method method_of(Method m) {
    switch (m) {
        case Method::XTT: return XR_METHOD_XTT;
        case Method::MLEM: return XR_METHOD_MLEM;
        case Method::ART: return XR_METHOD_ART;
        default: return XR_METHOD_FDK;
    }
}
inline xr_rotate rotate_of(Rotate r) { return r == Rotate::CW ? XR_ROTATE_CW : XR_ROTATE_CCW; }
inline std::vector<float *> ptrs(Volume<float> *v, int n) {
    std::vector<float *> p(n);
    for (int i = 0; i < n; i++) p[i] = v[i].get();
    return p;
}
inline void check_geom(const Geometry &g) {
    xr_scan s;
    check(xr_get_scan(need(), &s), "xr_get_scan");
    if (g.voxel != s.num_voxel || g.detect != s.num_detect || g.nProj != s.num_proj)
        throw Error(XR_ERR_ARG, "Geometry does not match the loaded settings");
}
}  // namespace xr

/* reconstruct.cuh:26-31 */
namespace IR {
inline void reconstruct(Volume<float> *sinogram, Volume<float> *voxel, const Geometry &geom, int epoch, int batch,
                        Rotate dir, Method method, float lambda = 1e-2) {
    xr::check_geom(geom);
    auto s = xr::ptrs(sinogram, NUM_PROJ_COND);
    auto v = xr::ptrs(voxel, NUM_PROJ_COND);
    xr::check(xr_ir_reconstruct(xr::need(), s.data(), v.data(), epoch, batch, xr::rotate_of(dir),
                                xr::method_of(method), lambda, nullptr),
              "IR::reconstruct");
}
}  // namespace IR

/* reconstruct.cuh:41-45 */
namespace XTT {
inline void reconstruct(Volume<float> *sinogram, Volume<float> *voxel, Volume<float> *md, const Geometry &geom,
                        int epoch, int batch, Rotate dir, Method method, float lambda = 1e-2) {
    xr::check_geom(geom);
    auto s = xr::ptrs(sinogram, NUM_PROJ_COND);
    auto v = xr::ptrs(voxel, NUM_BASIS_VECTOR);
    std::vector<float *> m;
    if (md) m = xr::ptrs(md, 3);
    xr::check(xr_xtt_reconstruct(xr::need(), s.data(), v.data(), md ? m.data() : nullptr, nullptr, epoch, batch,
                                 xr::rotate_of(dir), xr::method_of(method), lambda, nullptr),
              "XTT::reconstruct");
}

/* reconstruct.cuh:54-55: the fiber model, channel 0 updated, every channel
 * starting at 0.01; sinogram receives the last ratio images. */
inline void fiberModelReconstruct(Volume<float> *sinogram, Volume<float> *voxel, const Geometry &geom, int epoch,
                                  int batch, Rotate dir, Method method, float lambda = 1e-2) {
    xr::check_geom(geom);
    auto s = xr::ptrs(sinogram, NUM_PROJ_COND);
    auto v = xr::ptrs(voxel, NUM_BASIS_VECTOR);
    xr::check(xr_fiber_reconstruct(xr::need(), s.data(), v.data(), epoch, batch, xr::rotate_of(dir),
                                   xr::method_of(method), lambda, nullptr),
              "XTT::fiberModelReconstruct");
}
}  // namespace XTT

/* reconstruct.cuh:33-39 */
namespace FDK {
inline void reconstruct(Volume<float> *sinogram, Volume<float> *voxel, const Geometry &geom, Rotate dir) {
    xr::check_geom(geom);
    auto s = xr::ptrs(sinogram, NUM_PROJ_COND);
    auto v = xr::ptrs(voxel, NUM_PROJ_COND);
    xr::check(xr_fdk_reconstruct(xr::need(), s.data(), v.data(), xr::rotate_of(dir), XR_FILTER_REFERENCE),
              "FDK::reconstruct");
}
}  // namespace FDK

/* reconstruct.cuh:65 */
inline void forwardProjOnly(Volume<float> *sinogram, Volume<float> *voxel, const Geometry &geom, Rotate dir) {
    xr::check_geom(geom);
    auto s = xr::ptrs(sinogram, NUM_PROJ_COND);
    const float *v0 = voxel[0].get();
    xr::check(xr_forward_proj_only(xr::need(), &v0, s.data(), xr::rotate_of(dir)), "forwardProjOnly");
}

/* calcEigenVector, direction/src/pca.cu:12-55, one voxel on the host (FP64
 * cyclic Jacobi, Golub & Van Loan section 8.5). */
inline void calcEigenVector(const Volume<float> *ct, Volume<float> *md, Volume<float> *evalue, int x, int y,
                            int z) {
    double T[9] = {0}, mean = 0;
    for (int k = 0; k < NUM_BASIS_VECTOR; k++) {
        const double m = ct[k](x, y, z);
        const double s[3] = {m * basisVector[3 * k], m * basisVector[3 * k + 1], m * basisVector[3 * k + 2]};
        mean += m;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) T[3 * a + b] += s[a] * s[b];
    }
    mean /= NUM_BASIS_VECTOR;
    for (double &t : T) t /= NUM_BASIS_VECTOR;
    double V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int sweep = 0; sweep < 50; sweep++) {
        const double off = T[1] * T[1] + T[2] * T[2] + T[5] * T[5];
        const double dia = T[0] * T[0] + T[4] * T[4] + T[8] * T[8];
        if (off <= 1e-300 || off <= 1e-34 * dia) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                const double apq = T[3 * p + q];
                if (apq == 0.0) continue;
                const double th = (T[3 * q + q] - T[3 * p + p]) / (2.0 * apq);
                const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; k++) {
                    const double a = T[3 * k + p], b = T[3 * k + q];
                    T[3 * k + p] = c * a - s * b;
                    T[3 * k + q] = s * a + c * b;
                }
                for (int k = 0; k < 3; k++) {
                    const double a = T[3 * p + k], b = T[3 * q + k];
                    T[3 * p + k] = c * a - s * b;
                    T[3 * q + k] = s * a + c * b;
                }
                for (int k = 0; k < 3; k++) {
                    const double a = V[3 * k + p], b = V[3 * k + q];
                    V[3 * k + p] = c * a - s * b;
                    V[3 * k + q] = s * a + c * b;
                }
            }
    }
    int idx[3] = {0, 1, 2};
    const double w[3] = {T[0], T[4], T[8]};
    for (int a = 0; a < 3; a++)
        for (int b = a + 1; b < 3; b++)
            if (w[idx[b]] < w[idx[a]]) std::swap(idx[a], idx[b]);
    double v[3] = {V[idx[0]], V[3 + idx[0]], V[6 + idx[0]]};
    const double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double sg = (v[2] / n) >= 0 ? 1.0 : -1.0;
    for (int a = 0; a < 3; a++) md[a](x, y, z) = (float)(sg * mean * v[a] / n);
    const double tr = w[0] + w[1] + w[2];
    for (int a = 0; a < 3; a++) evalue[a](x, y, z) = (float)(w[idx[a]] / tr);
}

/* Every voxel at once, on the GPU. */
inline void calcEigenVectorAll(const Volume<float> *ct, Volume<float> *md, Volume<float> *evalue) {
    std::vector<const float *> c(NUM_BASIS_VECTOR);
    for (int k = 0; k < NUM_BASIS_VECTOR; k++) c[k] = ct[k].get();
    auto m = xr::ptrs(md, 3);
    std::vector<float *> e;
    if (evalue) e = xr::ptrs(evalue, 3);
    xr::check(xr_orientation(xr::need(), c.data(), m.data(), evalue ? e.data() : nullptr), "calcEigenVectorAll");
}

/* direction/src/pca.cu:67-83 (sizes must match the loaded settings). */
inline void calcAngleFromMD(const Volume<float> md[3], Volume<float> angle[2], int, int, int) {
    const float *m[3] = {md[0].get(), md[1].get(), md[2].get()};
    float *a[2] = {angle[0].get(), angle[1].get()};
    xr::check(xr_angle_from_md(xr::need(), m, a), "calcAngleFromMD");
}

/* direction/src/pca.cu:85-106 */
inline void directionNormalization(Volume<float> md[3]) {
    float *m[3] = {md[0].get(), md[1].get(), md[2].get()};
    xr::check(xr_direction_normalization(xr::need(), m), "directionNormalization");
}

/* solver/src/tvmin.cpp:6-98, on the GPU (device 0). */
inline void totalVariationMinimized(Volume<float> &vol, float rho, float lambda, int iter) {
    xr::check(xr_tv_minimize_host(0, vol.get(), vol.x(), vol.y(), vol.z(), rho, lambda, iter),
              "totalVariationMinimized");
}

/* reconstruct/src/quadfilt.cpp:11-134, on the GPU (device 0). */
inline void quadlicFormFilterCPU(Volume<float> voxel[3], Volume<float> *coefficient, float lambda) {
    float *v[3] = {voxel[0].get(), voxel[1].get(), voxel[2].get()};
    float *c[2] = {coefficient[0].get(), coefficient[1].get()};
    xr::check(xr_quad_form_filter_host(0, v, c, voxel[0].x(), voxel[0].y(), voxel[0].z(), lambda),
              "quadlicFormFilterCPU");
}

#endif /* XR_COMPAT_HPP */
