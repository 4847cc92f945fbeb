/* Stand-in for OpenMM's public Vec3 (openmm/Vec3.h), used to build and test the
 * CUDA kernel adapter in an environment without OpenMM.  With OpenMM present
 * the adapter compiles against OpenMM's own headers instead. */
#ifndef TDP_STANDIN_OPENMM_VEC3_H_
#define TDP_STANDIN_OPENMM_VEC3_H_
namespace OpenMM {
class Vec3 {
public:
    Vec3() { v[0] = v[1] = v[2] = 0.0; }
    Vec3(double x, double y, double z) { v[0] = x; v[1] = y; v[2] = z; }
    double operator[](int i) const { return v[i]; }
    double& operator[](int i) { return v[i]; }
    Vec3 operator+(const Vec3& o) const { return Vec3(v[0] + o[0], v[1] + o[1], v[2] + o[2]); }
    Vec3 operator-(const Vec3& o) const { return Vec3(v[0] - o[0], v[1] - o[1], v[2] - o[2]); }
    Vec3 operator*(double s) const { return Vec3(v[0] * s, v[1] * s, v[2] * s); }
    Vec3& operator+=(const Vec3& o) { v[0] += o[0]; v[1] += o[1]; v[2] += o[2]; return *this; }
    double dot(const Vec3& o) const { return v[0] * o[0] + v[1] * o[1] + v[2] * o[2]; }
private:
    double v[3];
};
}  // namespace OpenMM
#endif
