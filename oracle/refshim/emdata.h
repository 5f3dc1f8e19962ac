/*
 * Minimal stand-in for the EMAN2 headers that the reference's inserter source
 * (libEM/reconstructor_tools.cpp) includes.  TEST INFRASTRUCTURE ONLY: this
 * lets oracle/build_ref.sh compile the reference's own insert_pixel()
 * implementations and its EMData::add_complex_at_fast (libEM/emdata_core.h,
 * included verbatim from the reference tree inside the EMData class below)
 * into oracle/_ref/, so the C restatement in fr_oracle.c can be checked
 * against the reference's own arithmetic.  Everything here is new code that
 * supplies only the interfaces those two reference files use.
 */
#ifndef FR_REFSHIM_EMDATA_H
#define FR_REFSHIM_EMDATA_H
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

using std::string;
using std::vector;

namespace EMAN {

class EMData;

struct EMConsts {
  static const float I2G, I3G, I4G, I5G;
  static const double pi, deg2rad, rad2deg;
};

/* Util::fast_exp restates libEM/util.cpp:788-800 (table of exp(-i/50)). */
struct Util {
  static float fast_exp(const float &f) {
    static float mem[1000];
    static bool init = false;
    if (!init) { for (int i = 0; i < 1000; i++) mem[i] = (float)std::exp(-i / 50.0); init = true; }
    if (f > 0 || f < -19.98) return std::exp(f);
    int g = (int)(-f * 50.0 + 0.5);
    return mem[g];
  }
  static inline float hypot3sq(float x, float y, float z) { return (x * x + y * y + z * z); }
  static inline float hypot3(float x, float y, float z) { return std::sqrt(x * x + y * y + z * z); }
  static inline int fast_floor(float x) { if (x < 0) return ((int)x - 1); return (int)x; }
  static inline float square(float x) { return x * x; }
  template <class T> static inline T get_min(T a, T b) { return a < b ? a : b; }
  static float agauss(float, float, float, float, float) { std::abort(); }
  static void getBaldwinGridWeights(int, float, float, float, float) { std::abort(); }
  static vector<float> getBaldwinGridWeights(const int &, const float &, const float &, const float &, const float &, const float &) { std::abort(); }
};

struct NotExistingObjectException : std::runtime_error {
  NotExistingObjectException(const string &a, const string &b) : std::runtime_error(a + ": " + b) {}
};
struct OutofRangeException : std::runtime_error {
  OutofRangeException(int, int, int, const string &s) : std::runtime_error(s) {}
};

class EMObject {
 public:
  enum ObjectType { UNKNOWN, EMDATA, FLOAT_POINTER, INT, FLOAT };
  EMObject() {}
  EMObject(EMData *e) : emdata(e) {}
  EMObject(float *p) : fp(p) {}
  EMObject(int v) : iv(v) {}
  operator EMData *() const { return emdata; }
  operator float *() const { return fp; }
  operator int() const { return iv; }
  EMData *emdata = nullptr;
  float *fp = nullptr;
  int iv = 0;
};

class Dict {
 public:
  bool has_key(const string &k) const { return m.count(k) > 0; }
  EMObject &operator[](const string &k) { return m[k]; }
  EMObject operator[](const string &k) const { return m.at(k); }
  std::map<string, EMObject> m;
};

class TypeDict {
 public:
  void put(const string &, EMObject::ObjectType, const string & = "") {}
};

class FactoryBase {
 public:
  virtual ~FactoryBase() {}
  virtual string get_name() const = 0;
  virtual string get_desc() const = 0;
  void set_params(const Dict &d) { params = d; }
  Dict params;
};

template <class T> class Factory {
 public:
  Factory();
  template <class C> void force_add() {}
};

typedef int Vec3i[3];

class EMData {
 public:
  EMData() {}
  void set_volume(float *d, int x, int y, int z) {
    rdata = d; nx = x; ny = y; nz = z; nxy = (size_t)x * y; nxyz = nxy * z;
  }
  int get_xsize() const { return nx; }
  int get_ysize() const { return ny; }
  int get_zsize() const { return nz; }
  bool has_attr(const string &) const { return false; }
  EMObject get_attr(const string &) const { return EMObject(); }
  float *get_data() const { return rdata; }
  void update() {}

 private:
  float *rdata = nullptr;
  int nx = 0, ny = 0, nz = 0;
  size_t nxy = 0, nxyz = 0;
  int xoff = 0, yoff = 0, zoff = 0;

 public:
/* The reference's own EMData method fragment, included verbatim from the
 * reference tree (found through the -I path set by oracle/build_ref.sh). */
#include "emdata_core.h"
};

/* EMData::add_complex_at (libEM/emdata_core.cpp:251-295) is textually the
 * same algorithm as the inline add_complex_at_fast above; the stand-in
 * forwards to it. */
inline size_t EMData::add_complex_at(const int &x, const int &y, const int &z, const std::complex<float> &val) {
  return add_complex_at_fast(x, y, z, val);
}
inline size_t EMData::add_complex_at(int, int, int, const int &, const int &, const int &, const int &, const int &,
                                     const int &, const std::complex<float> &) { std::abort(); }
inline std::complex<float> EMData::get_complex_at(const int &, const int &, const int &) const { std::abort(); }

}  // namespace EMAN
#endif
