// spiffe_b200/csrc/geometry.cu -- define_geometry on the host.
//
// Boundary points become metal flags exactly as process_geometry_definition
// (geometry.c:132-362) and the drawing routines of grid_drawing.c make them:
// segments and arcs are sampled at half-cell steps and every sample marks
// its nearest node as surface (add_point, grid_drawing.c:445-486); vacuum is
// flood-filled from a seed (fill_in_drawing, :889-1084); leftover single
// rows on the region edges are trimmed (:1165-1190); then each metal node
// records which staggered field components it forces to zero and each row
// its last active node (geometry.c:319-362).  The sampling sequence,
// including its floating-point accumulation, is the reference's, because the
// flags decide every later field value.
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/spiffe_b200_constants.h"
#include "../../include/spiffe_b200.h"
#include "../../include/spiffe_b200_geometry.h"
#include "../../include/spiffe_b200_types.h"
#include "namelist.hpp"

extern "C" int spiffe_set_error(int code, const char *msg);

namespace {

struct Point {
  int type;
  double x, y, x0, y0, r, theta, a, b;
  double potential;
  short material, ramp_potential;
};

// The drawing state of grid_drawing.c (static there, a struct here).
struct Canvas {
  int nx, ny;
  double xmin, xmax, ymin, ymax, dx, dy, dtheta = 0;
  int16_t *lattice;
  double *potential;
  int16_t *material;
  std::vector<double> xb, yb;
  std::vector<long> ixb, iyb; // the node of each boundary point (ix_dbnd, iy_dbnd)
  std::vector<short> mb;      // that node's material (material_bnd)
  long n_outside = 0;
  bool vacuum_defined = false;
  int ix_vac = 0, iy_vac = 0;
  int stride() const { return ny + 1; }
  int16_t &L(int i, int j) { return lattice[(size_t)i * stride() + j]; }
  double &Pt(int i, int j) { return potential[(size_t)i * stride() + j]; }
  int16_t &Mt(int i, int j) { return material[(size_t)i * stride() + j]; }

  // add_point, grid_drawing.c:445-486
  void add_point(double x, double y, double pot, short mat)
  {
    if (!xb.empty() && xb.back() == x && yb.back() == y)
      return;
    const int i = (int)((x - xmin) / dx + 0.5), j = (int)((y - ymin) / dy + 0.5);
    short m = 0;
    if (i >= 0 && j >= 0 && i < nx && j < ny) {
      L(i, j) = SPIFFE_FL_IS_SURFACE;
      Pt(i, j) = pot;
      if (Mt(i, j) == 0)
        Mt(i, j) = mat;
      m = Mt(i, j);
    } else {
      n_outside++; // (the reference reads the material outside the lattice here)
    }
    xb.push_back(x);
    yb.push_back(y);
    ixb.push_back(i);
    iyb.push_back(j);
    mb.push_back(m);
  }

  // draw_line, grid_drawing.c:215-295
  void draw_line(double xi, double yi, double xf, double yf, double pot, short mat, double start_pot)
  {
    double slope, intercept, x, y, _dx, _dy, pot_slope;
    if (std::fabs(xi - xf) >= dx) {
      slope = (yf - yi) / (xf - xi);
      if (std::fabs(yf - yi) < dy / 1e6)
        slope = 0;
      intercept = yi - slope * xi;
      _dx = dx;
      if (std::fabs(slope * _dx) > std::fabs(dy))
        _dx = dy * .5 / std::fabs(slope);
      pot_slope = (pot - start_pot) / (xf - xi);
      _dx = 0.5 * _dx;
      if (xi <= xf) {
        x = xi;
        do {
          y = slope * x + intercept;
          add_point(x, y, start_pot + pot_slope * (x - xi), mat);
        } while ((x += _dx) <= xf);
      } else {
        x = xi;
        do {
          y = slope * x + intercept;
          add_point(x, y, start_pot + pot_slope * (x - xi), mat);
        } while ((x -= _dx) >= xf);
      }
      add_point(xf, yf, pot, mat);
    } else if (std::fabs(yi - yf) >= dy) {
      slope = (xf - xi) / (yf - yi);
      if (std::fabs(xf - xi) < dx / 1e6)
        slope = 0;
      intercept = xi - slope * yi;
      pot_slope = (pot - start_pot) / (yf - yi);
      _dy = dy * 0.5;
      if (yi <= yf) {
        y = yi;
        do {
          x = slope * y + intercept;
          add_point(x, y, start_pot + pot_slope * (y - yi), mat);
        } while ((y += _dy) <= yf);
      } else {
        y = yi;
        do {
          x = slope * y + intercept;
          add_point(x, y, start_pot + pot_slope * (y - yi), mat);
        } while ((y -= _dy) >= yf);
      }
      add_point(xf, yf, pot, mat);
    } else {
      add_point(xf, yf, pot, mat);
    }
  }

  // the arc sampler shared by draw_circle (:297-366) and draw_ellipse (:368-443)
  void arc(double xi, double yi, double xc, double yc, double a, double b, bool circle, double thetaf, double *xf,
           double *yf, double pot, short mat)
  {
    double theta = circle ? std::atan2(yi - yc, xi - xc) : std::atan2((yi - yc) / b, (xi - xc) / a);
    const bool sense = theta < thetaf;
    if (circle) {
      if (a != 0)
        dtheta = std::fmin(dx, dy) / a / 2;
      else if (dx < dy)
        dtheta = dx / (xmax - xmin) / 2;
      else
        dtheta = dy / (ymax - ymin) / 2;
    } else {
      dtheta = std::fmin(dx / a, dy / b) / 2;
    }
    double step;
    if (sense) {
      step = dtheta;
      while (theta > thetaf)
        theta -= SPIFFE_PIx2;
    } else {
      while (theta < thetaf)
        theta += SPIFFE_PIx2;
      step = -dtheta;
    }
    int n = (int)std::fabs((thetaf - theta) / step);
    if (n < 15) {
      n = 15;
      const double sgn = step > 0 ? 1 : (step < 0 ? -1 : 0);
      step = sgn * std::fabs(thetaf - theta) / n;
    }
    step *= 0.5;
    n *= 2;
    const double theta0 = theta;
    double x, y;
    for (int i = 1; i < n; i++) {
      x = xc + a * std::cos(theta);
      y = yc + b * std::sin(theta);
      add_point(x, y, pot, mat);
      theta = theta0 + i * step;
    }
    x = xc + a * std::cos((thetaf + theta) / 2);
    y = yc + b * std::sin((thetaf + theta) / 2);
    add_point(x, y, pot, mat);
    x = xc + a * std::cos(thetaf);
    y = yc + b * std::sin(thetaf);
    add_point(x, y, pot, mat);
    *xf = x;
    *yf = y;
  }

  // set_vacuum_point, grid_drawing.c:428-438
  void set_vacuum_point(double x, double y)
  {
    ix_vac = (int)((x - xmin) / dx + 0.5);
    iy_vac = (int)((y - ymin) / dy + 0.5);
    vacuum_defined = true;
    if (ix_vac < 0 || ix_vac >= nx || iy_vac < 0 || iy_vac >= ny)
      n_outside++;
  }

  // fill_in_drawing, grid_drawing.c:889-1084
  bool fill()
  {
    const int16_t V = SPIFFE_FL_IS_VACUUM;
    int i, j;
    if (!vacuum_defined) {
      for (i = 0; i < nx; i++)
        if (L(i, 0) && !L(i, 1))
          break;
      if (i == nx)
        return false;
      if (i > 0)
        L(i, 1) = V;
    } else {
      L(ix_vac, iy_vac) = V;
    }
    auto spread = [&](int a, int c) {
      long changed = 0;
      if (L(a, c) == V) {
        if (L(a, c + 1) == 0) { changed++; L(a, c + 1) = V; }
        if (L(a, c - 1) == 0) { changed++; L(a, c - 1) = V; }
        if (L(a + 1, c) == 0) { changed++; L(a + 1, c) = V; }
        if (L(a - 1, c) == 0) { changed++; L(a - 1, c) = V; }
      }
      return changed;
    };
    long changed = 1;
    while (changed) {
      changed = 0;
      for (i = 1; i < nx - 1; i++) {
        for (j = 1; j < ny - 1; j++)
          changed += spread(i, j);
        for (j = ny - 2; j > 0; j--)
          changed += spread(i, j);
      }
      for (i = nx - 2; i > 0; i--) {
        for (j = 1; j < ny - 1; j++)
          changed += spread(i, j);
        for (j = ny - 2; j > 0; j--)
          changed += spread(i, j);
      }
    }
    for (i = 0; i < nx; i++)
      for (j = 0; j < ny; j++) {
        if (L(i, j) == 0)
          L(i, j) = SPIFFE_FL_IS_INSIDE;
        else if (L(i, j) == V)
          L(i, j) = 0;
      }
    // interior nodes next to vacuum become surface, with their neighbours'
    // mean potential (the pass is serial and sees its own changes)
    for (i = 1; i < nx - 1; i++)
      for (j = 1; j < ny - 1; j++) {
        if (L(i, j) != SPIFFE_FL_IS_INSIDE)
          continue;
        int change = 0;
        long n_summed = 0;
        double sum = 0;
        for (int i1 = -1; i1 <= 1; i1++)
          for (int j1 = -1; j1 <= 1; j1++) {
            if (i1 == 0 && j1 == 0)
              continue;
            if (!L(i + i1, j + j1))
              change++;
            else if (L(i + i1, j + j1) == SPIFFE_FL_IS_SURFACE) {
              sum += Pt(i + i1, j + j1);
              n_summed++;
            }
          }
        if (change == 8)
          L(i, j) = 0;
        else if (change) {
          L(i, j) = SPIFFE_FL_IS_SURFACE;
          Pt(i, j) = n_summed ? sum / n_summed : 0;
        }
      }
    return true;
  }

  // trim_drawing, grid_drawing.c:1165-1190 (the top edge is not trimmed)
  void trim()
  {
    int i, j;
    for (j = 0; j < ny; j++)
      if (L(0, j) && !L(1, j))
        L(0, j) = 0;
    i = nx - 1;
    for (j = 0; j < ny; j++)
      if (L(i, j) && !L(i - 1, j))
        L(i, j) = 0;
    for (i = 0; i < nx; i++)
      if (L(i, 0) && !L(i, 1))
        L(i, 0) = 0;
  }
};

// ---------------------------------------------------------------- &po text

using spiffe_nl::NlEntry;
using spiffe_nl::next_block;

} // namespace

static int rasterise(const spiffe_geometry_options *o, const char *text, int16_t *flags, double *psi,
                     int16_t *material, Canvas &c);

extern "C" int spiffe_geometry_rasterise(const spiffe_geometry_options *o, const char *text, int16_t *flags,
                                         double *psi, int16_t *material)
{
  Canvas c;
  return rasterise(o, text, flags, psi, material, c);
}

// getBoundaryPoints, grid_drawing.c:541-760: the first run of consecutive
// boundary points of material `id`, as nodes without repeats; a corner node
// inserted wherever both indices change (passes repeat until none is added);
// then the side each segment faces.
static int boundary_points(Canvas &c, long id, std::vector<long> &iz, std::vector<long> &ir, std::vector<short> &dir)
{
  const long np = (long)c.mb.size();
  long i = 0;
  while (i < np && c.mb[(size_t)i] != id)
    i++;
  if (i == np)
    return 0;
  const long ip1 = i;
  for (i += 1; i < np; i++)
    if (c.mb[(size_t)i] != id)
      break;
  const long ip2 = i;
  for (i = ip1; i < ip2; i++) {
    if (i > ip1 && c.ixb[(size_t)i] == c.ixb[(size_t)i - 1] && c.iyb[(size_t)i] == c.iyb[(size_t)i - 1])
      continue;
    iz.push_back(c.ixb[(size_t)i]);
    ir.push_back(c.iyb[(size_t)i]);
  }
  auto in = [&](long a, long b) { return (c.L((int)a, (int)b) & SPIFFE_FL_IS_INSIDE) != 0; };
  auto surf = [&](long a, long b) { return (c.L((int)a, (int)b) & SPIFFE_FL_IS_SURFACE) != 0; };
  auto metal = [&](long a, long b) { return (c.L((int)a, (int)b) & SPIFFE_FL_IS_METAL) != 0; };
  long added;
  do {
    added = 0;
    for (i = 1; i < (long)iz.size(); i++) {
      const long iz0 = iz[(size_t)i - 1], iz1 = iz[(size_t)i], ir0 = ir[(size_t)i - 1], ir1 = ir[(size_t)i];
      if (iz0 == iz1 || ir0 == ir1)
        continue;
      long izn, irn;
      if (in(iz0, ir1)) {
        izn = iz0;
        irn = ir1;
      } else if (in(iz1, ir0)) {
        izn = iz1;
        irn = ir0;
      } else if (surf(iz0, ir1)) {
        izn = iz0;
        irn = ir1;
      } else if (surf(iz1, ir0)) {
        izn = iz1;
        irn = ir0;
      } else if (iz0 == 0) {
        izn = iz0;
        irn = ir1;
      } else {
        printf("boundary issue: (%ld, %ld) followed by (%ld, %ld)\n", iz0, ir0, iz1, ir1);
        continue;
      }
      iz.insert(iz.begin() + i, izn);
      ir.insert(ir.begin() + i, irn);
      i++; // the pass resumes after the old point, as the reference's does
      added++;
    }
    if (added)
      printf("Added %ld boundary points\n", added);
  } while (added);
  const long n = (long)iz.size(), nx = c.nx, ny = c.ny;
  dir.assign((size_t)n, 0);
  for (i = 1; i < n; i++) {
    const long z1 = iz[(size_t)i - 1], r1 = ir[(size_t)i - 1], z2 = iz[(size_t)i], r2 = ir[(size_t)i];
    short &d = dir[(size_t)i - 1];
    if (z1 == z2) { // a constant-z segment
      if (z1 == 0 || in(z1 - 1, r2) || in(z1 - 1, r1))
        d = SPIFFE_EMITS_RIGHT;
      else if (z2 == nx - 1 || in(z1 + 1, r2) || in(z1 + 1, r1))
        d = SPIFFE_EMITS_LEFT;
      else if (z1 > 1 && (in(z1 - 2, r2) || in(z1 - 2, r1)))
        d = SPIFFE_EMITS_RIGHT;
      else if (z1 < nx - 2 && (in(z1 + 2, r2) || in(z1 + 2, r1)))
        d = SPIFFE_EMITS_LEFT;
      else if (metal(z1 - 1, r2) || metal(z1 - 1, r1))
        d = SPIFFE_EMITS_RIGHT;
      else if (metal(z1 + 1, r2) || metal(z1 + 1, r1))
        d = SPIFFE_EMITS_LEFT;
      else {
        char buf[200];
        snprintf(buf, sizeof(buf), "Can't determine which way constant-z surface at z=%e, r=%e, iz=%ld, ir=%ld emits.",
                 z1 * c.dx + c.xmin, r1 * c.dy + c.ymin, z1, r1);
        return spiffe_set_error(SPIFFE_ERR_INVALID, buf);
      }
    } else if (r2 == r1) { // a constant-r segment
      if (r1 == 0 || in(z1, r1 - 1) || in(z2, r1 - 1))
        d = SPIFFE_EMITS_UP;
      else if (r2 == ny - 1 || in(z1, r1 + 1) || in(z2, r1 + 1))
        d = SPIFFE_EMITS_DOWN;
      else if (r1 > 1 && (in(z1, r1 - 2) || in(z2, r1 - 2)))
        d = SPIFFE_EMITS_UP;
      else if (r1 < ny - 2 && (in(z1, r1 + 2) || in(z2, r1 + 2)))
        d = SPIFFE_EMITS_DOWN;
      else if (metal(z1, r1 - 1) || metal(z2, r1 - 1))
        d = SPIFFE_EMITS_UP;
      else if (metal(z1, r1 + 1) || metal(z2, r1 + 1))
        d = SPIFFE_EMITS_DOWN;
      else {
        char buf[200];
        snprintf(buf, sizeof(buf), "Can't determine which way constant-r surface at z=%e, r=%e, iz=%ld, ir=%ld emits.",
                 z1 * c.dx + c.xmin, r1 * c.dy + c.ymin, z1, r1);
        return spiffe_set_error(SPIFFE_ERR_INVALID, buf);
      }
    } else if (i > 1) {
      d = dir[(size_t)i - 2];
    }
  }
  return (int)n;
}

extern "C" int spiffe_geometry_boundary_points(const spiffe_geometry_options *o, const char *text, int32_t material_id,
                                               int64_t max_points, int32_t *iz, int32_t *ir, int16_t *direction,
                                               int64_t *n_points)
{
  if (!o || !text || !n_points)
    return spiffe_set_error(SPIFFE_ERR_INVALID, "null argument");
  *n_points = 0;
  const size_t n = (size_t)(o->nz + 1) * (o->nr + 1);
  if (o->nz < 2 || o->nr < 2)
    return spiffe_set_error(SPIFFE_ERR_INVALID, "nz and nr must be greater than 2");
  std::vector<int16_t> flags(n), material(n);
  std::vector<double> psi(n);
  Canvas c;
  const int rc = rasterise(o, text, flags.data(), psi.data(), material.data(), c);
  if (rc)
    return rc;
  std::vector<long> vz, vr;
  std::vector<short> vd;
  const int np = boundary_points(c, material_id, vz, vr, vd);
  if (np < 0)
    return np;
  *n_points = np;
  if (!iz && !ir && !direction)
    return 0;
  if (np > max_points)
    return spiffe_set_error(SPIFFE_ERR_CAPACITY, "more boundary points than the buffers hold");
  for (int k = 0; k < np; k++) {
    if (iz)
      iz[k] = (int32_t)vz[(size_t)k];
    if (ir)
      ir[k] = (int32_t)vr[(size_t)k];
    if (direction)
      direction[k] = vd[(size_t)k];
  }
  return 0;
}

static int rasterise(const spiffe_geometry_options *o, const char *text, int16_t *flags, double *psi,
                     int16_t *material, Canvas &c)
{
  if (!o || !text || !flags || !psi)
    return spiffe_set_error(SPIFFE_ERR_INVALID, "null argument");
  if (o->nz < 2 || o->nr < 2)
    return spiffe_set_error(SPIFFE_ERR_INVALID, "nz and nr must be greater than 2");
  if (o->zmax <= o->zmin)
    return spiffe_set_error(SPIFFE_ERR_INVALID, "zmax must be greater than zmin");
  if (o->rmax <= 0)
    return spiffe_set_error(SPIFFE_ERR_INVALID, "rmax must be greater than 0");
  const int nz = o->nz, nr = o->nr;
  const size_t n = (size_t)(nz + 1) * (nr + 1);
  std::vector<int16_t> mat_store;
  if (!material) {
    mat_store.assign(n, 0);
    material = mat_store.data();
  }
  const double zr = o->zr_factor ? o->zr_factor : 1.0;

  // the &po points, geometry.c:133-210 (aovrb keeps its value from point to point)
  std::vector<Point> pts;
  double aovrb = 1;
  const std::string t(text);
  size_t pos = 0;
  std::string group, err;
  std::vector<NlEntry> ents;
  while (next_block(t, pos, group, ents, err)) {
    if (group != "point" && group != "po")
      return spiffe_set_error(SPIFFE_ERR_INVALID, "unrecognized namelist in boundary defintion");
    int nt = 1;
    short change_direction = 0, material_id = 0, ramp_potential = 0;
    double x = DBL_MAX, y = DBL_MAX, theta = DBL_MAX, x0 = 0, y0 = 0, r = 0, a = 0, b = 0, potential = 0;
    for (const NlEntry &e : ents) {
      const double v = std::strtod(e.value.c_str(), nullptr);
      if (e.name == "nt") nt = (int)v;
      else if (e.name == "x") x = v;
      else if (e.name == "y") y = v;
      else if (e.name == "x0") x0 = v;
      else if (e.name == "y0") y0 = v;
      else if (e.name == "r") r = v;
      else if (e.name == "theta") theta = v;
      else if (e.name == "a") a = v;
      else if (e.name == "b") b = v;
      else if (e.name == "aovrb") aovrb = v;
      else if (e.name == "potential") potential = v;
      else if (e.name == "material_id") material_id = (short)v;
      else if (e.name == "ramp_potential") ramp_potential = (short)v;
      else if (e.name == "change_direction") change_direction = (short)v;
      else
        return spiffe_set_error(SPIFFE_ERR_INVALID, ("unknown &po variable " + e.name).c_str());
    }
    if (theta != DBL_MAX)
      theta *= SPIFFE_PI / 180.0;
    if (pts.empty() && nt != 1)
      return spiffe_set_error(SPIFFE_ERR_INVALID, "first point in geometry definition must have nt=1");
    Point p{};
    p.type = nt;
    p.x = x * zr;
    p.y = y * zr;
    p.x0 = x0 * zr;
    p.y0 = y0 * zr;
    p.r = r * zr;
    a *= zr;
    b *= zr;
    if (x != DBL_MAX)
      x *= zr;
    if (y != DBL_MAX)
      y *= zr;
    if (nt == 2) {
      if (theta == DBL_MAX && (x == DBL_MAX || y == DBL_MAX))
        return spiffe_set_error(SPIFFE_ERR_INVALID, "If NT=2, must give theta or (x, y)");
      if (theta != DBL_MAX && (x != DBL_MAX || y != DBL_MAX))
        return spiffe_set_error(SPIFFE_ERR_INVALID, "If NT=2, must give theta or (x, y), not both");
      if (r == 0) {
        if (a == 0 && b == 0)
          return spiffe_set_error(SPIFFE_ERR_INVALID, "Can't have NT=2, R=0, A=0, and B=0");
        if (a == 0 || b == 0) {
          if (aovrb <= 0)
            return spiffe_set_error(SPIFFE_ERR_INVALID, "Can't have NT=2, R=0, AOVRB<=0 and A=0 or B=0");
          if (a == 0)
            a = b * aovrb;
          else
            b = a / aovrb;
        }
        if (theta == DBL_MAX)
          theta = std::atan2(y / b, x / a);
      } else if (theta == DBL_MAX) {
        theta = std::atan2(y, x);
      }
    }
    if (change_direction)
      theta = SPIFFE_PIx2 + theta;
    p.a = a;
    p.b = b;
    p.potential = potential;
    p.material = material_id;
    p.ramp_potential = ramp_potential;
    p.theta = theta;
    pts.push_back(p);
  }
  if (!err.empty())
    return spiffe_set_error(SPIFFE_ERR_INVALID, err.c_str());
  if (pts.empty())
    return spiffe_set_error(SPIFFE_ERR_INVALID, "too few boundary points in geometry file");

  // set_up_drawing, grid_drawing.c:157-196
  c.nx = nz;
  c.ny = nr;
  c.xmin = o->zmin;
  c.xmax = o->zmax;
  c.ymin = 0.0;
  c.ymax = o->rmax;
  c.dx = (c.xmax - c.xmin) / (c.nx - 1);
  c.dy = (c.ymax - c.ymin) / (c.ny - 1);
  c.lattice = flags;
  c.potential = psi;
  c.material = material;
  std::memset(flags, 0, n * sizeof(int16_t));
  std::memset(material, 0, n * sizeof(int16_t));
  std::memset(psi, 0, n * sizeof(double));

  // draw the boundary, geometry.c:217-289
  double xi = pts[0].x + pts[0].x0, yi = pts[0].y + pts[0].y0, xf, yf;
  c.add_point(xi, yi, pts[0].potential, pts[0].material);
  for (size_t k = 1; k < pts.size(); k++) {
    const Point &p = pts[k];
    switch (p.type) {
    case 1:
      xf = p.x + p.x0;
      yf = p.y + p.y0;
      c.draw_line(xi, yi, xf, yf, p.potential, p.material, p.ramp_potential ? pts[k - 1].potential : p.potential);
      if (c.n_outside) {
        char buf[256];
        snprintf(buf, sizeof(buf), "points on the boundary outside the simulation region for line (%g, %g) to (%g, %g)",
                 xi, yi, xf, yf);
        return spiffe_set_error(SPIFFE_ERR_INVALID, buf);
      }
      xi = xf;
      yi = yf;
      break;
    case 2:
      if (p.r != 0)
        c.arc(xi, yi, p.x0, p.y0, p.r, p.r, true, p.theta, &xf, &yf, p.potential, p.material);
      else
        c.arc(xi, yi, p.x0, p.y0, p.a, p.b, false, p.theta, &xf, &yf, p.potential, p.material);
      xi = xf;
      yi = yf;
      if (c.n_outside)
        return spiffe_set_error(SPIFFE_ERR_INVALID, "points on the boundary outside the simulation region for an arc");
      break;
    case 3:
      xi = p.x + p.x0;
      yi = p.y + p.y0;
      c.add_point(xi, yi, p.potential, p.material);
      break;
    case 4:
      c.set_vacuum_point(p.x + p.x0, p.y + p.y0);
      break;
    default:
      break;
    }
  }
  if (!c.fill())
    return spiffe_set_error(SPIFFE_ERR_INVALID,
                            "can't determine what points are in vacuum--use nt=4 point to mark a point that is in vacuum");
  c.trim();

  // field flags of metal nodes, geometry.c:319-350
  auto F = [&](int iz, int ir) -> int16_t & { return flags[(size_t)iz * (nr + 1) + ir]; };
  for (int iz = 0; iz < nz + 1; iz++)
    for (int ir = 0; ir < nr + 1; ir++) {
      if (!(F(iz, ir) & SPIFFE_FL_IS_METAL))
        continue;
      F(iz, ir) |= SPIFFE_FL_EPHI_ZERO;
      if (iz && F(iz - 1, ir) & SPIFFE_FL_IS_METAL)
        F(iz, ir) |= SPIFFE_FL_EZ_ZERO | SPIFFE_FL_BR_ZERO;
      if (ir == 0 || (ir && F(iz, ir - 1) & SPIFFE_FL_IS_METAL))
        F(iz, ir) |= SPIFFE_FL_ER_ZERO | SPIFFE_FL_BZ_ZERO;
      if (iz && F(iz - 1, ir) & SPIFFE_FL_IS_METAL &&
          (ir == 0 || (F(iz, ir - 1) & SPIFFE_FL_IS_METAL && F(iz - 1, ir - 1) & SPIFFE_FL_IS_METAL)))
        F(iz, ir) |= SPIFFE_FL_BPHI_ZERO;
    }
  // last active node of each row, geometry.c:352-362
  for (int ir = 0; ir < nr; ir++) {
    int iz = nz - 1;
    while (iz >= 0 && F(iz, ir) & SPIFFE_FL_IS_INSIDE)
      iz--;
    if (iz != 0 && (iz += 1) < nz - 1)
      F(iz, ir) |= SPIFFE_FL_LAST_ACTIVE_PT;
  }
  return 0;
}
