/* Minimal stand-in for OpenMM's public Vec3 type (three doubles with the
 * arithmetic the OpenMM API documents).  Written for this repository so the
 * reference plugin's physics source can be compiled as a CPU oracle without an
 * OpenMM installation.  Test infrastructure only. */
#ifndef TDP_SHIM_OPENMM_VEC3_H_
#define TDP_SHIM_OPENMM_VEC3_H_
#include <cassert>
#include <ostream>
namespace OpenMM {
class Vec3 {
public:
    Vec3() { v[0] = v[1] = v[2] = 0.0; }
    Vec3(double x, double y, double z) { v[0] = x; v[1] = y; v[2] = z; }
    double operator[](int i) const { return v[i]; }
    double& operator[](int i) { return v[i]; }
    bool operator==(const Vec3& o) const { return v[0] == o[0] && v[1] == o[1] && v[2] == o[2]; }
    bool operator!=(const Vec3& o) const { return !(*this == o); }
    Vec3 operator+() const { return *this; }
    Vec3 operator-() const { return Vec3(-v[0], -v[1], -v[2]); }
    Vec3 operator+(const Vec3& o) const { return Vec3(v[0] + o[0], v[1] + o[1], v[2] + o[2]); }
    Vec3 operator-(const Vec3& o) const { return Vec3(v[0] - o[0], v[1] - o[1], v[2] - o[2]); }
    Vec3 operator*(double s) const { return Vec3(v[0] * s, v[1] * s, v[2] * s); }
    Vec3 operator/(double s) const { double r = 1.0 / s; return Vec3(v[0] * r, v[1] * r, v[2] * r); }
    Vec3& operator+=(const Vec3& o) { v[0] += o[0]; v[1] += o[1]; v[2] += o[2]; return *this; }
    Vec3& operator-=(const Vec3& o) { v[0] -= o[0]; v[1] -= o[1]; v[2] -= o[2]; return *this; }
    Vec3& operator*=(double s) { v[0] *= s; v[1] *= s; v[2] *= s; return *this; }
    Vec3& operator/=(double s) { double r = 1.0 / s; v[0] *= r; v[1] *= r; v[2] *= r; return *this; }
    double dot(const Vec3& o) const { return v[0] * o[0] + v[1] * o[1] + v[2] * o[2]; }
    Vec3 cross(const Vec3& o) const {
        return Vec3(v[1] * o[2] - v[2] * o[1], v[2] * o[0] - v[0] * o[2], v[0] * o[1] - v[1] * o[0]);
    }
private:
    double v[3];
};
static inline Vec3 operator*(double s, const Vec3& a) { return a * s; }
template <class CHAR, class TRAITS>
std::basic_ostream<CHAR, TRAITS>& operator<<(std::basic_ostream<CHAR, TRAITS>& o, const Vec3& v) {
    o << '[' << v[0] << ", " << v[1] << ", " << v[2] << ']';
    return o;
}
}  // namespace OpenMM
#endif
