// Magnetic-field maps read from files into the grid form of srs_field (host code).
//
// Formats of the reference (TField3D_Grid.cc), each read with the same stream operations so that
// every sample is the same double:
//   OSCARS      regular 1/2/3-D grid, 10-line header (:318-509; here read_oscars)
//   OSCARS1D..  irregular samples along one axis, columns named in the format string, regridded at
//               10000 points per metre by linear interpolation (:533-812)
//   SRW         regular grid, header values behind the comment character (:836-1000)
//   SPECTRA     regular grid centred on 0, steps in mm (:1002-1148)
// and maps interpolated between several OSCARS files by a parameter such as an undulator gap
// (:1150-1446).  Sample values are rotated as the reference rotates them; the point rotation and the
// translation are applied at evaluation.
//
// Where the reference reads past an array, uses an uninitialised value it does not define or aborts
// the process (`throw;` outside a handler), this returns an error instead: a file ending before its
// header says, header values that differ between interpolated files, a parameter outside the mapping,
// more OSCARS1D scale factors than columns.  One of its values is kept as the reference (built with
// zero-initialised locals) computes it: interpolating at exactly the first mapping parameter gives NaN
// (the "before" index is never set, so the slope is 0/0).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {
namespace {

constexpr const char *kImportError = "Could not import magnetic field.  Check 'ifile' and 'iformat' are correct";

V3 rotated(double x, double y, double z, const double r[3]) {
  V3 v = v3(x, y, z);
  rotate_xyz(v, r);  // TVector3D::RotateSelfXYZ
  return v;
}

void grid_descriptor(srs_field &f, const double start[3], const double step[3], const int64_t n[3],
                     const double rot[3], const double trans[3]) {
  std::memset(&f, 0, sizeof f);
  f.kind = SRS_FIELD_GRID;
  for (int k = 0; k < 3; ++k) {
    f.start[k] = start[k];
    f.step[k] = step[k];
    f.n[k] = n[k];
    f.rotations[k] = rot[k];
    f.translation[k] = trans[k];
  }
}

std::string upper_case(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), ::toupper);
  return s;
}

// OSCARS format: a comment line, 9 header values (start, step, n per axis), then one "fx fy fz" line
// per sample in ix, iy, iz order; scale = (step x, y, z, field x, y, z) factors, the map kept
// centred where it was (TField3D_Grid.cc:318-509).
srs_status read_oscars(const std::string &path, const double rot[3], const double trans[3], const double *scale,
                       int nscale, srs_field &f, std::vector<double> &data) {
  std::ifstream fi(path);
  if (!fi) return fail(SRS_ERR_IO, kImportError);
  std::string L;
  std::getline(fi, L);  // comment line
  double hv[9];
  for (int k = 0; k < 9; ++k) {
    if (!std::getline(fi, L)) return fail(SRS_ERR_IO, "cannot read header value");
    std::istringstream S(L);
    S >> hv[k];
    if (S.fail()) return fail(SRS_ERR_IO, "cannot read header value");
  }
  const int NX = (int)hv[2], NY = (int)hv[5], NZ = (int)hv[8];
  const double XStepIN = hv[1], YStepIN = hv[4], ZStepIN = hv[7];
  const double XStep = nscale > 0 ? XStepIN * scale[0] : XStepIN;
  const double YStep = nscale > 1 ? YStepIN * scale[1] : YStepIN;
  const double ZStep = nscale > 2 ? ZStepIN * scale[2] : ZStepIN;
  const double FxS = nscale > 3 ? scale[3] : 1, FyS = nscale > 4 ? scale[4] : 1, FzS = nscale > 5 ? scale[5] : 1;
  const double MiddleX = hv[0] + XStepIN * (NX - 1) / 2., XStart = MiddleX - XStep * (NX - 1) / 2.;
  const double MiddleY = hv[3] + YStepIN * (NY - 1) / 2., YStart = MiddleY - YStep * (NY - 1) / 2.;
  const double MiddleZ = hv[6] + ZStepIN * (NZ - 1) / 2., ZStart = MiddleZ - ZStep * (NZ - 1) / 2.;
  if (NX < 1 || NY < 1 || NZ < 1) return fail(SRS_ERR_RANGE, "invalid number of points in at least one dimension");
  if (NX == 1 && NY == 1 && NZ == 1) return fail(SRS_ERR_RANGE, "invalid dimensions");
  const size_t n = (size_t)NX * NY * NZ;
  data.resize(3 * n);
  std::istringstream S;
  for (size_t i = 0; i < n; ++i) {
    std::getline(fi, L);
    if (fi.eof() && L.empty()) return fail(SRS_ERR_IO, "error reading file.  Check format");
    double fx, fy, fz;
    S.clear();
    S.str(L);
    S >> fx >> fy >> fz;
    if (S.fail()) return fail(SRS_ERR_IO, "error reading file.  Check format");
    if (FxS != 1) fx *= FxS;
    if (FyS != 1) fy *= FyS;
    if (FzS != 1) fz *= FzS;
    const V3 F = rotated(fx, fy, fz, rot);
    data[3 * i] = F.x;
    data[3 * i + 1] = F.y;
    data[3 * i + 2] = F.z;
  }
  const double start[3] = {XStart, YStart, ZStart}, step[3] = {XStep, YStep, ZStep};
  const int64_t nn[3] = {NX, NY, NZ};
  grid_descriptor(f, start, step, nn, rot, trans);
  return SRS_OK;
}

// OSCARS1D: the format string after "OSCARS1D" names the columns (one of X Y Z, and any of Bx/Ex/Fx,
// By/Ey/Fy, Bz/Ez/Fz, in file order); the first line is a comment, blank lines and lines starting
// with '#' are skipped, scale factors multiply the columns in order; the samples, sorted by position,
// are resampled on (size_t)((last - first) * 10000) points by linear interpolation between the
// neighbouring samples (TField3D_Grid.cc:533-812).
srs_status read_oscars1d(const std::string &path, const std::string &format, const double rot[3],
                         const double trans[3], const double *scale, int nscale, srs_field &f,
                         std::vector<double> &data) {
  std::ifstream fi(path);
  if (!fi) return fail(SRS_ERR_IO, kImportError);
  std::vector<int> order(4, -1);
  std::istringstream s(std::string(format.begin() + 8, format.end()));
  std::string c, axis;
  int index = 0, xdim = 0, fdim = 0;
  bool hasf[4] = {false, false, false, false};
  while (s >> c) {
    if (index > 3) return fail(SRS_ERR_RANGE, "spatial or B-field dimensions are too large(index>3)");
    if (c == "X" || c == "Y" || c == "Z") {
      axis = c;
      ++xdim;
      order[index++] = 0;
    } else if (c == "Bx" || c == "Ex" || c == "Fx") {
      hasf[1] = true;
      ++fdim;
      order[index++] = 1;
    } else if (c == "By" || c == "Ey" || c == "Fy") {
      hasf[2] = true;
      ++fdim;
      order[index++] = 2;
    } else if (c == "Bz" || c == "Ez" || c == "Fz") {
      hasf[3] = true;
      ++fdim;
      order[index++] = 3;
    } else {
      return fail(SRS_ERR_INVALID, "only excepts X Y Z Bx By Bz");
    }
  }
  const int ncol = xdim + fdim;
  if (xdim != 1) return fail(SRS_ERR_RANGE, "spatial or B-field dimensions are too large");
  if (nscale > ncol) return fail(SRS_ERR_RANGE, "more scale factors than columns");
  std::string L;
  std::getline(fi, L);  // comment line
  std::vector<std::array<double, 4>> in;
  std::istringstream S;
  while (std::getline(fi, L)) {
    const size_t first = L.find_first_not_of(" \t");
    if (first == std::string::npos || L[first] == '#') continue;
    S.clear();
    S.str(L);
    double value[4] = {0, 0, 0, 0};
    for (int i = 0; i < ncol; ++i) {
      S >> value[order[i]];
      if (S.fail()) return fail(SRS_ERR_IO, "something is incorrect with data format or iformat string");
    }
    for (int i = 0; i < nscale && i < 4; ++i) value[order[i]] *= scale[i];
    in.push_back({{value[0], value[1], value[2], value[3]}});
  }
  std::sort(in.begin(), in.end(),
            [](const std::array<double, 4> &a, const std::array<double, 4> &b) { return a[0] < b[0]; });
  if (in.size() < 2) return fail(SRS_ERR_RANGE, "not enough data points");
  const double First = in.front()[0], Last = in.back()[0];
  const int kPointsPerMeter = 10000;
  const size_t NPoints = (size_t)((Last - First) * kPointsPerMeter);
  if (NPoints < 2) return fail(SRS_ERR_RANGE, "invalid dimensions");
  const double StepSize = (Last - First) / (double)(NPoints - 1);
  data.resize(3 * NPoints);
  size_t minbin = 0, after = 0, before = 0;
  for (size_t i = 0; i != NPoints; ++i) {
    const double z = i * StepSize + First;
    for (size_t j = minbin + 1; j != in.size(); ++j) {
      if (in[j][0] > z) {  // the first sample past z; past the last sample the previous pair is kept
        after = j;
        before = j - 1;
        minbin = j - 1;
        break;
      }
    }
    double nb[4] = {0, 0, 0, 0};
    for (int k = 1; k < 4; ++k) {
      if (!hasf[k]) continue;
      const double slope = (in[after][k] - in[before][k]) / (in[after][0] - in[before][0]);
      nb[k] = in[before][k] + (z - in[before][0]) * slope;
    }
    const V3 F = rotated(nb[1], nb[2], nb[3], rot);
    data[3 * i] = F.x;
    data[3 * i + 1] = F.y;
    data[3 * i + 2] = F.z;
  }
  double start[3] = {0, 0, 0}, step[3] = {0, 0, 0};
  int64_t nn[3] = {1, 1, 1};
  const int a = axis == "X" ? 0 : axis == "Y" ? 1 : 2;
  start[a] = First;
  step[a] = StepSize;
  nn[a] = (int64_t)NPoints;
  grid_descriptor(f, start, step, nn, rot, trans);
  return SRS_OK;
}

// SRW: a comment line, then 9 header lines "#value" (start, step, n per axis), then "fx fy fz" per
// sample in ix, iy, iz order; no scaling (TField3D_Grid.cc:282-310, 836-1000).
srs_status read_srw(const std::string &path, const double rot[3], const double trans[3], srs_field &f,
                    std::vector<double> &data) {
  std::ifstream fi(path);
  if (!fi) return fail(SRS_ERR_IO, "cannot open file for reading SRW format");
  std::string L;
  std::getline(fi, L);  // comment line
  double hv[9];
  for (int k = 0; k < 9; ++k) {
    std::getline(fi, L);
    std::istringstream S(L);
    char cc = 0;
    S.get(cc);
    if (cc != '#') return fail(SRS_ERR_IO, "something is wrong with the comment character, it was not seen");
    double v = 0;
    S >> v;  // a value that does not read is 0, as the reference's stream leaves it
    if (S.bad()) return fail(SRS_ERR_IO, "cannot read header value SRW format");
    hv[k] = S.fail() ? 0.0 : v;
  }
  const int NX = (int)hv[2], NY = (int)hv[5], NZ = (int)hv[8];
  if (NX < 1 || NY < 1 || NZ < 1) return fail(SRS_ERR_RANGE, "invalid dimensions");
  if (NX == 1 && NY == 1 && NZ == 1) return fail(SRS_ERR_RANGE, "invalid dimensions");
  const size_t n = (size_t)NX * NY * NZ;
  data.resize(3 * n);
  std::istringstream S;
  for (size_t i = 0; i < n; ++i) {
    std::getline(fi, L);
    double fx, fy, fz;
    S.clear();
    S.str(L);
    S >> fx >> fy >> fz;
    if (S.fail() || fi.fail()) return fail(SRS_ERR_IO, "input file stream failure");
    const V3 F = rotated(fx, fy, fz, rot);
    data[3 * i] = F.x;
    data[3 * i + 1] = F.y;
    data[3 * i + 2] = F.z;
  }
  const double start[3] = {hv[0], hv[3], hv[6]}, step[3] = {hv[1], hv[4], hv[7]};
  const int64_t nn[3] = {NX, NY, NZ};
  grid_descriptor(f, start, step, nn, rot, trans);
  return SRS_OK;
}

// SPECTRA: a comment line, "xstep ystep zstep nx ny nz" with steps in mm, then "fx fy fz" per sample;
// the grid is centred on 0; a sample line that ends the file without a newline is an error, as in the
// reference (TField3D_Grid.cc:1002-1148).
srs_status read_spectra(const std::string &path, const double rot[3], const double trans[3], srs_field &f,
                        std::vector<double> &data) {
  std::ifstream fi(path);
  if (!fi) return fail(SRS_ERR_IO, "cannot open file");
  std::string L;
  std::getline(fi, L);  // comment line
  std::getline(fi, L);
  std::istringstream H(L);
  double step[3] = {0, 0, 0};
  int NX = 0, NY = 0, NZ = 0;
  H >> step[0] >> step[1] >> step[2] >> NX >> NY >> NZ;
  if (H.bad()) return fail(SRS_ERR_IO, "file stream failure");
  step[0] /= 1000.;
  step[1] /= 1000.;
  step[2] /= 1000.;
  if (NX < 1 || NY < 1 || NZ < 1) return fail(SRS_ERR_RANGE, "invalid number of points in at least one dimension");
  if (NX == 1 && NY == 1 && NZ == 1) return fail(SRS_ERR_RANGE, "invalid dimensions");
  const double start[3] = {-(step[0] * (NX - 1)) / 2, -(step[1] * (NY - 1)) / 2, -(step[2] * (NZ - 1)) / 2};
  const size_t n = (size_t)NX * NY * NZ;
  data.resize(3 * n);
  std::istringstream S;
  for (size_t i = 0; i < n; ++i) {
    std::getline(fi, L);
    if (fi.eof()) return fail(SRS_ERR_IO, "file stream failure");
    double fx, fy, fz;
    S.clear();
    S.str(L);
    S >> fx >> fy >> fz;
    if (S.fail()) return fail(SRS_ERR_IO, "file stream failure");
    const V3 F = rotated(fx, fy, fz, rot);
    data[3 * i] = F.x;
    data[3 * i + 1] = F.y;
    data[3 * i + 2] = F.z;
  }
  const int64_t nn[3] = {NX, NY, NZ};
  grid_descriptor(f, start, step, nn, rot, trans);
  return SRS_OK;
}

// Linear interpolation in the parameter between the two mapping entries around it
// (TField3D_Grid::InterpolateFields, :1382-1420); "before" starts at 0 as the reference's unset
// index reads when locals are zero-initialised.
V3 interpolate(const std::vector<double> &P, const std::vector<V3> &F, double p) {
  size_t before = 0, after = 0;
  for (size_t i = 0; i != P.size(); ++i) {
    if (P[i] < p) {
      before = i;
    } else {
      after = i;
      break;
    }
  }
  const double d = p - P[before], den = P[after] - P[before];
  const V3 slope = v3((F[after].x - F[before].x) / den, (F[after].y - F[before].y) / den,
                      (F[after].z - F[before].z) / den);
  return v3(F[before].x + slope.x * d, F[before].y + slope.y * d, F[before].z + slope.z * d);
}

}  // namespace

srs_status read_field_file(const std::string &path, const std::string &format, const double rot[3],
                           const double trans[3], const double *scale, int nscale, srs_field &f,
                           std::vector<double> &data) {
  // TField3D_Grid::TField3D_Grid (:25-45) with OSCARSSR::AddMagneticField's format check (:68-90)
  const std::string u = upper_case(format);
  if (u == "OSCARS") return read_oscars(path, rot, trans, scale, nscale, f, data);
  if (u.size() > 8 && u.compare(0, 8, "OSCARS1D") == 0)
    return read_oscars1d(path, format, rot, trans, scale, nscale, f, data);
  if (u == "SRW") return read_srw(path, rot, trans, f, data);
  if (u == "SPECTRA") return read_spectra(path, rot, trans, f, data);
  return fail(SRS_ERR_INVALID, kImportError);
}

srs_status read_field_interpolated(std::vector<std::pair<double, std::string>> mapping, const std::string &format,
                                   double parameter, const double rot[3], const double trans[3],
                                   const double *scale, int nscale, srs_field &f, std::vector<double> &data) {
  // TField3D_Grid::InterpolateFromFiles (:1150-1380): OSCARS-format files with identical headers
  if (upper_case(format) != "OSCARS") return fail(SRS_ERR_INVALID, "only OSCARS-format files can be interpolated");
  if (mapping.size() < 2) return fail(SRS_ERR_RANGE, "at least two files are needed");
  std::sort(mapping.begin(), mapping.end(),
            [](const std::pair<double, std::string> &a, const std::pair<double, std::string> &b) {
              return a.first < b.first;
            });
  if (!(parameter >= mapping.front().first && parameter <= mapping.back().first))
    return fail(SRS_ERR_RANGE, "parameter outside of the mapping range");
  std::vector<double> P;
  std::vector<std::ifstream> in(mapping.size());
  for (size_t i = 0; i < mapping.size(); ++i) {
    P.push_back(mapping[i].first);
    in[i].open(mapping[i].second);
    if (!in[i]) return fail(SRS_ERR_IO, "cannot open file for reading");
  }
  std::string L;
  double hv[10];
  for (int ih = 0; ih < 10; ++ih) {
    for (size_t i = 0; i < in.size(); ++i) {
      std::getline(in[i], L);
      std::istringstream S(L);
      double v = 0;
      S >> v;
      if (S.bad()) return fail(SRS_ERR_IO, "cannot read header value");
      if (S.fail()) v = 0;
      if (i == 0) hv[ih] = v;
      else if (v != hv[ih]) return fail(SRS_ERR_INVALID, "the files' headers differ");
    }
  }
  const int NX = (int)hv[3], NY = (int)hv[6], NZ = (int)hv[9];
  const double XStep = nscale > 0 ? hv[2] * scale[0] : hv[2];
  const double YStep = nscale > 1 ? hv[5] * scale[1] : hv[5];
  const double ZStep = nscale > 2 ? hv[8] * scale[2] : hv[8];
  const double FxS = nscale > 3 ? scale[3] : 1, FyS = nscale > 4 ? scale[4] : 1, FzS = nscale > 5 ? scale[5] : 1;
  const double MiddleX = hv[1] + hv[2] * (NX - 1) / 2., XStart = MiddleX - XStep * (NX - 1) / 2.;
  const double MiddleY = hv[4] + hv[5] * (NY - 1) / 2., YStart = MiddleY - YStep * (NY - 1) / 2.;
  const double MiddleZ = hv[7] + hv[8] * (NZ - 1) / 2., ZStart = MiddleZ - ZStep * (NZ - 1) / 2.;
  if (NX < 1 || NY < 1 || NZ < 1) return fail(SRS_ERR_RANGE, "invalid number of points in at least one dimension");
  if (NX == 1 && NY == 1 && NZ == 1) return fail(SRS_ERR_RANGE, "invalid dimensions");
  const size_t n = (size_t)NX * NY * NZ;
  data.resize(3 * n);
  std::vector<V3> F(in.size());
  std::istringstream S;
  for (size_t s = 0; s < n; ++s) {
    for (size_t i = 0; i < in.size(); ++i) {
      std::getline(in[i], L);
      if (in[i].eof()) return fail(SRS_ERR_IO, "error reading file.  Check format");
      double fx, fy, fz;
      S.clear();
      S.str(L);
      S >> fx >> fy >> fz;
      if (FxS != 1) fx *= FxS;
      if (FyS != 1) fy *= FyS;
      if (FzS != 1) fz *= FzS;
      if (S.fail()) return fail(SRS_ERR_IO, "error reading file.  Check format");
      F[i] = v3(fx, fy, fz);
    }
    const V3 I = interpolate(P, F, parameter);
    const V3 R = rotated(I.x, I.y, I.z, rot);
    data[3 * s] = R.x;
    data[3 * s + 1] = R.y;
    data[3 * s + 2] = R.z;
  }
  const double start[3] = {XStart, YStart, ZStart}, step[3] = {XStep, YStep, ZStep};
  const int64_t nn[3] = {NX, NY, NZ};
  grid_descriptor(f, start, step, nn, rot, trans);
  return SRS_OK;
}

}  // namespace srs
