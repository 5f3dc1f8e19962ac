/*
 * ref_driver.cpp -- C entry points around the reference's own pixel
 * inserters (libEM/reconstructor_tools.cpp, compiled from the reference tree
 * by build_ref.sh together with this file).  TEST INFRASTRUCTURE ONLY: used by
 * tests/test_oracle_ref.py to pin the C restatement in fr_oracle.c against the
 * reference's insert_pixel() and EMData::add_complex_at_fast arithmetic.
 */
#include "reconstructor_tools.h"

using namespace EMAN;

/* EMConsts values as defined in libEM/emobject.cpp:53-59 (that file itself
 * is not compiled here). */
const float EMConsts::I2G = (float)(4.0 / (M_PI * M_PI));
const float EMConsts::I3G = (float)(6.4 / (M_PI * M_PI));
const float EMConsts::I4G = (float)(8.8 / (M_PI * M_PI));
const float EMConsts::I5G = (float)(10.4 / (M_PI * M_PI));
const double EMConsts::pi = 3.141592653589793238462643383279502884197169399;
const double EMConsts::deg2rad = pi / 180.0;
const double EMConsts::rad2deg = 180.0 / pi;

extern "C" {

/* Runs n calls of the reference inserter `mode` ("nearest_neighbor",
 * "gauss_2", "gauss_5", "trilinear") on a full (N+2)xNxN complex volume
 * `data` and its (N/2+1)xNxN weight volume `norm`.  px[n*6] holds
 * (xx, yy, zz, re, im, weight) per call. */
int ref_insert_pixels(const char *mode, float *data, float *norm, int N, const float *px, long n) {
  EMData vol;
  vol.set_volume(data, N + 2, N, N);
  FourierPixelInserter3D *ins = nullptr;
  string m(mode);
  if (m == "nearest_neighbor") ins = new FourierInserter3DMode1();
  else if (m == "gauss_2") ins = new FourierInserter3DMode2();
  else if (m == "gauss_5") ins = new FourierInserter3DMode5();
  else if (m == "trilinear") ins = new FourierInserter3DMode2l();
  else return -1;
  Dict d;
  d["data"] = EMObject(&vol);
  d["norm"] = EMObject(norm);
  ins->set_params(d);
  ins->init();
  for (long i = 0; i < n; i++) {
    const float *p = px + 6 * i;
    ins->insert_pixel(p[0], p[1], p[2], std::complex<float>(p[3], p[4]), p[5]);
  }
  delete ins;
  return 0;
}

/* The reference's EMData::add_complex_at_fast on its own, for index checks:
 * returns the float index it reports (nxyz when rejected). */
long ref_add_complex_at_fast(float *data, int N, int x, int y, int z, float re, float im) {
  EMData vol;
  vol.set_volume(data, N + 2, N, N);
  return (long)vol.add_complex_at_fast(x, y, z, std::complex<float>(re, im));
}

}
