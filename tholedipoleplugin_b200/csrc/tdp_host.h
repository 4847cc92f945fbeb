// tdp_host.h -- host-side pieces shared by the single-system handle
// (tdp_capi.cu) and the cluster batch (tdp_batch_capi.cu): error type,
// device allocation, input validation, the covalent scale table and the
// Thole damping radius.
#pragma once

#include "tholedipole_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

namespace tdp {

struct TdpError {
    int code;
    std::string msg;
};

#define TDP_CUDA(call)                                                                                      \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess)                                                                              \
            throw ::tdp::TdpError{TDP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)};       \
    } while (0)

template <class T>
inline T* dalloc(size_t count, std::vector<void*>& owned) {
    void* p = nullptr;
    if (count == 0) count = 1;
    TDP_CUDA(cudaMalloc(&p, count * sizeof(T)));
    owned.push_back(p);
    TDP_CUDA(cudaMemset(p, 0, count * sizeof(T)));
    return static_cast<T*>(p);
}

inline void upload(void* dst, const void* src, size_t bytes) {
    if (bytes) TDP_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
}

// Validation: TholeDipoleForceImpl::initialize (openmmapi/src/TholeDipoleForceImpl.cpp:52-108)
// plus the inputs on which the reference dereferences null or out-of-range
// memory (rotation of an atom with Z set and no X atom, RTDF.cpp:556-568).
inline void validate_axes(int n, const int32_t* types, const int32_t* zs, const int32_t* xs, const int32_t* ys) {
    for (int i = 0; i < n; i++) {
        int t = types[i], z = zs[i], x = xs[i], y = ys[i];
        char buf[256];
        if (t < TDP_ZTHENX || t > TDP_NO_AXIS_TYPE) {
            snprintf(buf, sizeof buf,
                     "TholeDipoleForce: axis type=%d not currently handled - only axisTypes[ 0, 1, 2, 3, 4, 5] "
                     "(ZThenX, Bisector, Z-Bisect, ThreeFold, ZOnly, NoAxisType) currently handled.",
                     t);
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, buf};
        }
        if (t != TDP_NO_AXIS_TYPE && (z < 0 || z >= n)) {
            snprintf(buf, sizeof buf, "TholeDipoleForce: invalid z axis particle: %d", z);
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, buf};
        }
        if (t != TDP_NO_AXIS_TYPE && t != TDP_ZONLY && (x < 0 || x >= n)) {
            snprintf(buf, sizeof buf, "TholeDipoleForce: invalid x axis particle: %d", x);
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, buf};
        }
        if ((t == TDP_ZBISECT || t == TDP_THREEFOLD) && (y < 0 || y >= n)) {
            snprintf(buf, sizeof buf, "TholeDipoleForce: invalid y axis particle: %d", y);
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, buf};
        }
        if (z >= n || x >= n || y >= n) {
            snprintf(buf, sizeof buf, "TholeDipoleForce: axis particle index out of range for particle %d", i);
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, buf};
        }
        if (z >= 0 && z != i && t != TDP_ZONLY && x < 0) {
            snprintf(buf, sizeof buf,
                     "TholeDipoleForce: particle %d has a z axis particle but no x axis particle (the reference "
                     "platform dereferences a null particle here)",
                     i);
            throw TdpError{TDP_ERR_INVALID_ARGUMENT, buf};
        }
    }
}

// Covalent scales (RTDF.cpp:609-644): pair (i<j) takes _mScale[pos] for j at
// list position pos of Covalent12(i) and _iScale[pos] for Covalent13(i), the
// last occurrence winning; only the lower-index atom's lists count.  Lists of
// more than five entries index past the scale tables in the reference and are
// rejected.  Returns, per atom, its partners whose (M, I) differ from (1, 1),
// each pair listed on both atoms.
inline std::vector<std::vector<std::tuple<int, double, double>>> covalent_exceptions(
    int n, const int32_t* off12, const int32_t* atoms12, const int32_t* off13, const int32_t* atoms13) {
    static const double kM[5] = {0.0, 0.0, 0.0, 0.5, 1.0};
    static const double kI[5] = {0.0, 1.0, 1.0, 1.0, 1.0};
    std::map<std::pair<int, int>, std::pair<double, double>> scales;
    for (int i = 0; i < n; i++) {
        for (int list = 0; list < 2; list++) {
            const int32_t* off = list == 0 ? off12 : off13;
            const int32_t* atoms = list == 0 ? atoms12 : atoms13;
            if (!off) continue;
            int b = off[i], e = off[i + 1];
            if (e - b > 5) {
                char buf[200];
                snprintf(buf, sizeof buf,
                         "TholeDipoleForce: particle %d has %d Covalent1%d entries; only five scale factors exist", i,
                         e - b, list == 0 ? 2 : 3);
                throw TdpError{TDP_ERR_INVALID_ARGUMENT, buf};
            }
            for (int p = b; p < e; p++) {
                int j = atoms[p];
                if (j <= i || j >= n) continue;
                auto it = scales.find({i, j});
                if (it == scales.end()) it = scales.insert({{i, j}, {1.0, 1.0}}).first;
                if (list == 0) it->second.first = kM[p - b];
                else it->second.second = kI[p - b];
            }
        }
    }
    std::vector<std::vector<std::tuple<int, double, double>>> exc(n);
    for (auto& kv : scales) {
        double m = kv.second.first, s = kv.second.second;
        if (m == 1.0 && s == 1.0) continue;
        exc[kv.first.first].push_back(std::make_tuple(kv.first.second, m, s));
        exc[kv.first.second].push_back(std::make_tuple(kv.first.first, m, s));
    }
    return exc;
}

// Squared distance beyond which the Thole factors are exactly 1:
// a*u^3 < 50 needs r < t_i t_j (50/min(t_i,t_j))^(1/3) <= tmax^(5/3) 50^(1/3).
inline double damp_radius2(const std::vector<double>& thole) {
    double tmax = 0.0;
    bool negative = false;
    for (double t : thole) {
        if (t < 0.0 || std::isnan(t)) negative = true;
        tmax = std::max(tmax, t);
    }
    if (negative) return INFINITY;
    if (tmax == 0.0) return 0.0;
    double r = std::pow(tmax, 5.0 / 3.0) * std::cbrt(50.0) * 1.001;
    return r * r;
}

// Torque-mapping users (RTDF.cpp:915-1115): for every atom a, the frames
// (atom i, role) that send it force; role 0 I, 1 Z, 2 X, 3 Y.  CSR by atom.
inline void torque_users(int n, const std::vector<int>& axis, std::vector<int>& off, std::vector<int2>& flat) {
    std::vector<std::vector<std::pair<int, int>>> users(n);
    for (int i = 0; i < n; i++) {
        int t = axis[4 * i], z = axis[4 * i + 1], x = axis[4 * i + 2], y = axis[4 * i + 3];
        if (t == TDP_NO_AXIS_TYPE) continue;
        users[i].push_back({i, 0});
        users[z].push_back({i, 1});
        if (t != TDP_ZONLY && x >= 0) users[x].push_back({i, 2});
        if ((t == TDP_ZBISECT || t == TDP_THREEFOLD) && y > -1) users[y].push_back({i, 3});
    }
    off.assign(n + 1, 0);
    flat.clear();
    for (int a = 0; a < n; a++) {
        for (auto& u : users[a]) flat.push_back(make_int2(u.first, u.second));
        off[a + 1] = (int)flat.size();
    }
}

}  // namespace tdp
