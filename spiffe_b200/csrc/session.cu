// spiffe_b200/csrc/session.cu -- spiffe's namelist command surface (host
// code; the commands and their mapping are listed in spiffe_b200_session.h).
//
// Each command restates the reference's command processor: defaults, checks
// and derived quantities follow the cited file:line; the physics then runs in
// the device loop of runtime.cu.  Errors return a negative code with the
// reference's message where the reference bombs.
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/spiffe_b200.h"
#include "../../include/spiffe_b200_constants.h"
#include "../../include/spiffe_b200_geometry.h"
#include "../../include/spiffe_b200_session.h"
#include "../../include/spiffe_b200_types.h"
#include "namelist.hpp"
#include "onaxis.hpp"
#include "sdds.hpp"

extern "C" int spiffe_set_error(int code, const char *msg);
extern "C" int spiffe_cathode_check(const spiffe_mesh *mesh, const spiffe_cathode_options *o);

namespace {

int serr(int code, const char *fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return spiffe_set_error(code, buf);
}

#define S_TRY(x)        \
  do {                  \
    const int rc_ = (x); \
    if (rc_ < 0)        \
      return rc_;       \
  } while (0)

std::string lower(std::string s)
{
  for (auto &c : s)
    c = (char)std::tolower((unsigned char)c);
  return s;
}

// match_string as spiffe uses it: an exact (case-insensitive) match, else
// the one entry the value abbreviates; -1 if none or ambiguous.
int match(const std::string &v, const std::vector<std::string> &names)
{
  const std::string lv = lower(v);
  for (size_t i = 0; i < names.size(); i++)
    if (lower(names[i]) == lv)
      return (int)i;
  int hit = -1;
  for (size_t i = 0; i < names.size(); i++)
    if (!lv.empty() && lower(names[i]).compare(0, lv.size(), lv) == 0) {
      if (hit >= 0)
        return -1;
      hit = (int)i;
    }
  return hit;
}

// compose_filename: "%s" in a name becomes the rootname.
std::string compose(const std::string &name, const std::string &root)
{
  const size_t p = name.find("%s");
  if (p == std::string::npos)
    return name;
  return name.substr(0, p) + root + name.substr(p + 2);
}

bool read_text(const std::string &path, std::string &out, std::string &err)
{
  FILE *fp = std::fopen(path.c_str(), "rb");
  if (!fp) {
    err = "unable to open " + path;
    return false;
  }
  out.clear();
  char buf[1 << 14];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), fp)) > 0)
    out.append(buf, n);
  std::fclose(fp);
  return true;
}

// The variables of one command.  Getters leave the default when a variable
// is absent; unused() names a variable no getter asked for (the reference's
// namelist processor rejects unknown variables).
struct Args {
  std::string group;
  std::vector<spiffe_nl::NlEntry> e;
  std::vector<char> used;
  std::string bad;

  int find(const char *name)
  {
    int k = -1;
    for (size_t i = 0; i < e.size(); i++)
      if (e[i].name == name) {
        used[i] = 1;
        k = (int)i;
      }
    return k;
  }
  void num(const char *name, double &v)
  {
    const int k = find(name);
    if (k < 0)
      return;
    const char *s = e[(size_t)k].value.c_str();
    char *end = nullptr;
    const double x = std::strtod(s, &end);
    while (end && *end && std::isspace((unsigned char)*end))
      end++;
    if (end == s || (end && *end))
      bad = "invalid value \"" + e[(size_t)k].value + "\" for " + name;
    else
      v = x;
  }
  template <class I> void integer(const char *name, I &v)
  {
    double x = (double)v;
    num(name, x);
    v = (I)x;
  }
  bool str(const char *name, std::string &v)
  {
    const int k = find(name);
    if (k < 0)
      return false;
    v = e[(size_t)k].value;
    return true;
  }
  int finish()
  {
    if (!bad.empty())
      return serr(SPIFFE_ERR_INVALID, "%s: %s", group.c_str(), bad.c_str());
    for (size_t i = 0; i < e.size(); i++)
      if (!used[i])
        return serr(SPIFFE_ERR_INVALID, "unknown variable %s in namelist %s", e[i].name.c_str(), group.c_str());
    return 0;
  }
};

struct SessionScreen {
  std::string filename;
  double z = 0;
  int direction = 1;
  spiffe_sdds::Writer out;
  bool on_device = false;
};

struct SessionCathode {
  spiffe_cathode_options o{};
  std::vector<double> t, A;
  bool on_device = false;
};

// one define_field_sampling definition and its file
struct SessionSampling {
  spiffe_sample_options o{};
  std::string path;
  int32_t index = -1; // on the device
  spiffe_sdds::Writer out;
  bool opened = false;
  std::vector<double> seq_t, seq_v[3]; // a time sequence's rows so far
  double seq_param[3] = {0, 0, 0};
};

// one define_emitter definition with its surface and profile
struct SessionEmitter {
  spiffe_emitter_options o{};
  std::vector<int32_t> iz, ir;
  std::vector<int16_t> dir;
  std::vector<double> t, A;
  bool on_device = false;
};

// one define_secondary_emission definition with its yield table
struct SessionSecondary {
  spiffe_secondary_options o{};
  std::vector<double> E, Y;
  bool on_device = false;
  spiffe_sdds::Writer log_out; // log_file, open from the definition on
};

// one add_on_axis_fields definition: the file's columns and the namelist
// values, given to the device instance when it exists
struct SessionOnAxis {
  std::vector<double> z, Ez;
  double z_offset = 0, Ez_peak = 0, frequency = 0, phase = 0; // phase in radians once read
  long long order = 3;
  bool on_device = false;
};

struct SessionAntenna {
  int direction = 0;
  long istart = 0, iend = 0, iposition = 0;
  double current = 0, frequency = 0, phase = 0;
  std::vector<double> t, W;
  bool on_device = false;
};

// FIELD_SAVING, spiffe.h; step_interval/start_step/save_index are set on
// the first save_fields call (field_saving.c:63-70)
struct FieldSaving {
  bool defined = false;
  std::string filename;
  double time_interval = -1, start_time = 0;
  long long save_before_exiting = 0;
  long long step_interval = -1, start_step = -1;
  long long save_index = -1;
  spiffe_sdds::Writer out;
};

// SNAPSHOT and FIELD_OUTPUT, spiffe.h:320-398; step_interval/start_step are
// set on the first call of the integration loop (snapshots.c:60-63,
// field_output.c:58-61)
struct BeamSnapshots {
  bool defined = false;
  std::string filename;
  double time_interval = 0, start_time = 0;
  long long step_interval = -1, start_step = -1, index = -1;
  spiffe_sdds::Writer out;
};

struct FieldOutput {
  bool defined = false;
  std::string filename;
  double time_interval = 0, start_time = 0;
  long long z_interval = 1, r_interval = 1, exclude_imposed = 0, separate_imposed = 0;
  long long step_interval = -1, start_step = -1, index = -1;
  spiffe_sdds::Writer out;
};

// the shared schedule test of the diagnostics (field_saving.c:138-147,
// snapshots.c:79-80, field_output.c:126-127)
bool due(long long step, long long start_step, long long step_interval)
{
  return step >= start_step && (step_interval == 0 || (step - start_step) % step_interval == 0);
}

// the first step at or after `from` the schedule selects
long long next_due(long long from, long long start_step, long long step_interval)
{
  long long j = from > start_step ? from : start_step;
  if (step_interval > 0) {
    const long long r = (j - start_step) % step_interval;
    if (r)
      j += step_interval - r;
  }
  return j;
}

const char *const kFieldNames[] = {"Ez",  "Er",  "Bphi",      "Bphi2",     "Jz",         "Jr",        "Ephi",
                                   "Jphi", "Br", "Br2",       "Bz",        "Bz2",        "EzImposed", "ErImposed",
                                   "PsiImposed", "BzImposed", "BrImposed", "Psi",        "Q"};

double **slot(spiffe_field_set &f, const std::string &n)
{
#define SLOT(x) \
  if (n == #x)  \
    return &f.x;
  SLOT(Ez) SLOT(Er) SLOT(Bphi) SLOT(Bphi2) SLOT(Jz) SLOT(Jr) SLOT(Ephi) SLOT(Jphi) SLOT(Br) SLOT(Br2) SLOT(Bz)
  SLOT(Bz2) SLOT(EzImposed) SLOT(ErImposed) SLOT(PsiImposed) SLOT(BzImposed) SLOT(BrImposed) SLOT(Psi) SLOT(Q)
#undef SLOT
  return nullptr;
}

} // namespace

struct spiffe_session {
  int precision = SPIFFE_PRECISION_F64;
  std::string rootname = "spiffe";
  std::string run_name = "spiffe"; // EM_problem->run_name: the input file (spiffe.c:204)
  int verbose = 1;
  int deposit_order = 1;
  long long particle_capacity = 1 << 16, screen_capacity = 1 << 20, flush_steps = 512;
  int compaction = -1, screen_momentum = -1;
  int poisson_solver = -1; // SPIFFE_POISSON_* of the split form (-1: the instance's default)

  bool have_geometry = false;
  spiffe_mesh mesh{};
  std::vector<int16_t> flags;
  std::map<std::string, std::vector<double>> a; // mesh arrays by FieldSet name

  std::vector<SessionCathode> cathodes;
  std::vector<SessionSecondary> secondaries;
  std::vector<SessionEmitter> emitters;
  std::vector<SessionSampling> samplings;
  spiffe_geometry_options geo_opts{}; // define_geometry's drawing, for the emitters' surfaces
  std::string geo_text;
  std::vector<int16_t> material; // define_geometry's surface materials (materialID)
  std::vector<SessionAntenna> antennas;
  std::vector<SessionOnAxis> onaxis;
  std::vector<OnAxisProfile> onaxis_prepared; // for the fields_used output
  // integrate's status_output: the rows so far (the file is rewritten whole
  // after each row, so it is a complete one-page table at every point)
  bool status_on = false;
  std::string status_path;
  std::vector<std::vector<double>> status_cols;
  std::vector<std::vector<int32_t>> status_counts;
  int64_t status_old_np = 0;
  // integrate's lost_particles file (setUpLostParticleFile, advance_particles.c:577-603)
  bool lost_on = false;
  std::string lost_path;
  spiffe_sdds::Writer lost_out;
  bool translate_on = false, translate_set = false; // translate: the moving window
  double z_trigger = 0;
  std::vector<SessionScreen> screens;
  bool test_beam = false;
  spiffe_test_beam_options tb{};
  double tb_z_force = 0, tb_r_force = 0, tb_z_decel = DBL_MAX, tb_r_decel = DBL_MAX;
  bool pc_defined = false;
  spiffe_poisson_options pc{};
  FieldSaving saving;
  BeamSnapshots snapshots;
  FieldOutput field_output;
  // integrate.nl variables the reference does not reset between commands
  double ramp_time = 0, flat_top_time = 1;
  long long auto_max_dt = 0;

  spiffe_gpu_instance *inst = nullptr;
  long long steps = 0;

  void say(const char *fmt, ...)
  {
    if (!verbose)
      return;
    va_list ap;
    va_start(ap, fmt);
    std::vfprintf(stdout, fmt, ap);
    va_end(ap);
    std::fflush(stdout);
  }
  void warn(const char *fmt, ...)
  {
    va_list ap;
    va_start(ap, fmt);
    std::fputs("spiffe_b200 warning: ", stderr);
    std::vfprintf(stderr, fmt, ap);
    std::fputc('\n', stderr);
    va_end(ap);
  }
  size_t nodes() const { return (size_t)(mesh.nz + 1) * (size_t)(mesh.nr + 1); }
  std::vector<double> &arr(const char *n) { return a[n]; }
  bool has(const char *n) const { return a.count(n) != 0; }

  spiffe_field_set host_set(bool all = true)
  {
    spiffe_field_set f{};
    for (auto &kv : a)
      if (all || kv.first != "Psi")
        *slot(f, kv.first) = kv.second.data();
    return f;
  }
  // the device holds the current fields and mesh once an instance exists
  int pull()
  {
    if (!inst)
      return 0;
    S_TRY(spiffe_gpu_get_mesh(inst, &mesh));
    spiffe_field_set f = host_set();
    return spiffe_gpu_download_fields(inst, &f);
  }
  int push_fields(const std::vector<const char *> &names)
  {
    if (!inst)
      return 0;
    S_TRY(spiffe_gpu_set_mesh(inst, &mesh));
    spiffe_field_set f{};
    for (const char *n : names)
      if (has(n))
        *slot(f, n) = a[n].data();
    return spiffe_gpu_upload_fields(inst, &f);
  }

  int cmd_geometry(Args &g);
  int cmd_constant_fields(Args &g);
  int cmd_solenoid(Args &g);
  int cmd_cathode(Args &g);
  int cmd_antenna(Args &g);
  int cmd_on_axis_fields(Args &g);
  int cmd_translate(Args &g);
  int cmd_screen(Args &g);
  int cmd_secondary_emission(Args &g);
  int cmd_emitter(Args &g);
  int cmd_field_sampling(Args &g);
  int flush_samples();
  int cmd_test_beam(Args &g);
  int cmd_poisson(Args &g);
  int cmd_load_fields(Args &g);
  int cmd_field_saving(Args &g);
  int cmd_snapshots(Args &g);
  int cmd_field_output(Args &g);
  int cmd_integrate(Args &g);
  int execute(const std::string &text);

  int ensure_instance();
  int save_fields(long long step, double time, bool final_call);
  int take_snapshot(long long step, double time);
  int output_fields(long long step, double time);
  int flush_screens(long long step, double time);
  int flush_lost();
  int flush_secondary_logs();
  int status(long long step, double time);
  int write_status();
};

// ------------------------------------------------------------ define_geometry

// process_geometry_definition, geometry.c:21-131 (the drawing, :132-362, is
// spiffe_geometry_rasterise)
int spiffe_session::cmd_geometry(Args &g)
{
  long long nz = 0, nr = 0, include_te = 0, exclude_tm = 0, print_grids = 0, rad_i = 1, lon_i = 1, rad_s = 0,
            lon_s = 0;
  long long off[6] = {0, 0, 0, 0, 0, 0};
  double zmin = 0, zmax = 0, rmax = 0, zr_factor = 1;
  std::string boundary, root, lower_bc = "Dirichlet", upper_bc = "Neumann", right_bc = "Neumann",
                             left_bc = "Neumann", out;
  g.integer("nz", nz);
  g.integer("nr", nr);
  g.num("zmin", zmin);
  g.num("zmax", zmax);
  g.num("rmax", rmax);
  g.num("zr_factor", zr_factor);
  const bool have_root = g.str("rootname", root);
  const bool have_boundary = g.str("boundary", boundary);
  for (const char *o : {"boundary_output", "urmel_boundary_output", "discrete_boundary_output", "interior_points"})
    if (g.str(o, out))
      warn("define_geometry: %s is not written", o);
  g.str("lower", lower_bc);
  g.str("upper", upper_bc);
  g.str("right", right_bc);
  g.str("left", left_bc);
  g.integer("include_te_fields", include_te);
  g.integer("exclude_tm_fields", exclude_tm);
  // turn_off_* in the order of spiffe_mesh.turn_off: Ez, Er, Ephi, Bz, Br, Bphi
  g.integer("turn_off_ez", off[0]);
  g.integer("turn_off_er", off[1]);
  g.integer("turn_off_ephi", off[2]);
  g.integer("turn_off_bz", off[3]);
  g.integer("turn_off_br", off[4]);
  g.integer("turn_off_bphi", off[5]);
  g.integer("print_grids", print_grids);
  g.integer("radial_interpolation", rad_i);
  g.integer("longitudinal_interpolation", lon_i);
  g.integer("radial_smearing", rad_s);
  g.integer("longitudinal_smearing", lon_s);
  S_TRY(g.finish());
  if (inst)
    return serr(SPIFFE_ERR_UNSUPPORTED, "define_geometry after integrate is not supported");
  if (have_root)
    rootname = root;
  if (!have_boundary)
    return serr(SPIFFE_ERR_INVALID, "no boundary-points file named");
  if (nz < 2 || nr < 2)
    return serr(SPIFFE_ERR_INVALID, "nz and nr must be greater than 2");
  if (zmax <= zmin)
    return serr(SPIFFE_ERR_INVALID, "zmax must be greater than zmin");
  if (rmax <= 0)
    return serr(SPIFFE_ERR_INVALID, "rmax must be greater than 0");
  const std::vector<std::string> types = {"Dirichlet", "Neumann"}; // SPIFFE_DIRICHLET, SPIFFE_NEUMANN
  spiffe_mesh m{};
  if ((m.lower_bc = match(lower_bc, types)) < 0)
    return serr(SPIFFE_ERR_INVALID, "unrecognized boundary condition for lower boundary");
  if (m.lower_bc == SPIFFE_NEUMANN)
    return serr(SPIFFE_ERR_INVALID, "Neumann boundary conditions are meaningless on the lower boundary");
  if ((m.upper_bc = match(upper_bc, types)) < 0)
    return serr(SPIFFE_ERR_INVALID, "unrecognized boundary condition for upper boundary");
  if (m.upper_bc == SPIFFE_DIRICHLET)
    return serr(SPIFFE_ERR_INVALID, "Dirichlet boundary conditions are not implemented for the upper boundary");
  if ((m.right_bc = match(right_bc, types)) < 0)
    return serr(SPIFFE_ERR_INVALID, "unrecognized boundary condition for right boundary");
  if ((m.left_bc = match(left_bc, types)) < 0)
    return serr(SPIFFE_ERR_INVALID, "unrecognized boundary condition for left boundary");
  m.nz = (int32_t)nz;
  m.nr = (int32_t)nr;
  m.zmin = zmin;
  m.zmax = zmax;
  m.rmax = rmax;
  m.dz = (zmax - zmin) / (nz - 1);
  m.dr = rmax / (nr - 1);
  m.modes = (rad_i ? SPIFFE_FL_RADIAL_INTERP : 0) + (lon_i ? SPIFFE_FL_LONGIT_INTERP : 0) +
            (rad_s ? SPIFFE_FL_RADIAL_SMEAR : 0) + (lon_s ? SPIFFE_FL_LONGIT_SMEAR : 0);
  if (!exclude_tm)
    m.modes |= SPIFFE_FL_TM_FIELDS;
  if (include_te)
    m.modes |= SPIFFE_FL_TE_FIELDS;
  if (!(m.modes & (SPIFFE_FL_TM_FIELDS | SPIFFE_FL_TE_FIELDS)))
    warn("all rf fields are disabled");
  for (int i = 0; i < 6; i++)
    m.turn_off[i] = (int16_t)off[i];
  m.imposed_flat_top_time = 1;

  std::string text, err;
  if (!read_text(boundary, text, err))
    return serr(SPIFFE_ERR_INVALID, "define_geometry: %s", err.c_str());
  mesh = m;
  const size_t n = nodes();
  flags.assign(n, 0);
  material.assign(n, 0);
  a.clear();
  a["PsiImposed"].assign(n, 0.0);
  spiffe_geometry_options go{m.nz, m.nr, zmin, zmax, rmax, zr_factor};
  S_TRY(spiffe_geometry_rasterise(&go, text.c_str(), flags.data(), a["PsiImposed"].data(), material.data()));
  geo_opts = go;
  geo_text = text;
  // the arrays of geometry.c:78-116 that the device problem holds
  for (const char *x : {"EzImposed", "ErImposed", "Q", "Jz"})
    a[x].assign(n, 0.0);
  if (m.modes & SPIFFE_FL_TM_FIELDS)
    for (const char *x : {"Ez", "Er", "Jr", "Bphi", "Bphi2", "Psi"})
      a[x].assign(n, 0.0);
  if (m.modes & SPIFFE_FL_TE_FIELDS)
    for (const char *x : {"Ephi", "Jphi", "Bz", "Br", "Bz2", "Br2"})
      a[x].assign(n, 0.0);
  have_geometry = true;
  say("geometry: %d x %d nodes, dz=%.6e m, dr=%.6e m\n", m.nz, m.nr, m.dz, m.dr);
  return 0;
}

// set_constant_fields, constant_fields.c:18-39
int spiffe_session::cmd_constant_fields(Args &g)
{
  double Ez = 0, Er = 0, Ephi = 0, Bz = 0, Br = 0, Bphi = 0;
  g.num("ez", Ez);
  g.num("er", Er);
  g.num("ephi", Ephi);
  g.num("bz", Bz);
  g.num("br", Br);
  g.num("bphi", Bphi);
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "can't set constant fields before geometry is defined");
  if (inst)
    S_TRY(spiffe_gpu_get_mesh(inst, &mesh));
  mesh.constant_E[0] = Ez;
  mesh.constant_E[1] = Er;
  mesh.constant_E[2] = Ephi;
  mesh.constant_B[0] = Bz;
  mesh.constant_B[1] = Br;
  mesh.constant_B[2] = Bphi;
  if (inst)
    S_TRY(spiffe_gpu_set_mesh(inst, &mesh));
  return 0;
}

// process_solenoid_definition, solenoid.c:18-117
int spiffe_session::cmd_solenoid(Args &g)
{
  spiffe_solenoid_options o{};
  o.turns = 1;
  std::string out;
  g.num("radius", o.radius);
  g.num("evaluation_radius_limit", o.evaluation_radius_limit);
  g.num("z_start", o.z_start);
  g.num("z_end", o.z_end);
  g.num("current", o.current);
  g.num("bz_peak", o.Bz_peak);
  g.integer("turns", o.turns);
  g.integer("symmetry", o.symmetry);
  if (g.str("field_output", out))
    warn("define_solenoid: field_output is not written");
  g.integer("bucking", o.bucking);
  g.num("z_buck", o.z_buck);
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "can't define a solenoid before geometry is set up");
  if (inst)
    S_TRY(spiffe_gpu_get_mesh(inst, &mesh));
  if (!has("BzImposed")) {
    a["BzImposed"].assign(nodes(), 0.0);
    a["BrImposed"].assign(nodes(), 0.0);
  }
  double cur = 0;
  S_TRY(spiffe_solenoid_add(&mesh, &o, a["BzImposed"].data(), a["BrImposed"].data(), &cur));
  if (o.bucking)
    say("Bucking coil current set to %e\n", cur);
  mesh.has_solenoid = 1;
  return push_fields({"BzImposed", "BrImposed"});
}

// ------------------------------------------------------------- define_cathode

// process_cathode_definition, cathode.c:21-237 (the device loop holds the
// cathode; its checks are spiffe_cathode_check)
int spiffe_session::cmd_cathode(Args &g)
{
  spiffe_cathode_options o{};
  o.stiffness = 1;
  o.zoned_emission = 1;
  o.random_number_seed = 987654321;
  o.field_emission_beta = 1;
  long long add_thermal = 0, determine_temperature = 0, halton_dt = 0, halton_r = 0;
  double focal_length = 0;
  std::string profile, tname, fname, log;
  g.num("z_position", o.z_position);
  g.num("inner_radius", o.inner_radius);
  g.num("outer_radius", o.outer_radius);
  g.num("current_density", o.current_density);
  g.num("temperature", o.temperature);
  g.num("work_function", o.work_function);
  g.integer("field_emission", o.field_emission);
  g.integer("add_thermal_velocities", add_thermal);
  g.num("field_emission_beta", o.field_emission_beta);
  g.integer("determine_temperature", determine_temperature);
  g.num("electrons_per_macroparticle", o.electrons_per_macroparticle);
  g.num("start_time", o.start_time);
  g.num("stop_time", o.stop_time);
  g.integer("autophase", o.autophase);
  g.num("time_offset", o.time_offset);
  g.num("number_per_step", o.number_per_step);
  g.num("initial_pz", o.initial_pz);
  g.num("initial_omega", o.initial_omega);
  g.num("focal_length", focal_length); // declared by cathode.nl, read by no code
  g.num("stiffness", o.stiffness);
  g.integer("discretize_radii", o.discretize_radii);
  g.integer("random_number_seed", o.random_number_seed);
  g.integer("distribution_correction_interval", o.distribution_correction_interval);
  g.integer("spread_over_dt", o.spread_over_dt);
  g.integer("zoned_emission", o.zoned_emission);
  g.integer("halton_radix_dt", halton_dt);
  g.integer("halton_radix_r", halton_r);
  const bool have_profile = g.str("profile", profile);
  g.str("profile_time_name", tname);
  g.str("profile_factor_name", fname);
  if (g.str("emission_log", log))
    warn("define_cathode: emission_log is not written");
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "define_cathode before define_geometry");
  if (test_beam)
    return serr(SPIFFE_ERR_INVALID, "can't do both cathode and test particles");
  // cathode.c:50-62, the combinations spiffe_cathode_check does not see
  if (o.field_emission && (determine_temperature || o.current_density || have_profile))
    return serr(SPIFFE_ERR_INVALID, "field_emission is incompatible with determine_temperature, current_density, and profile");
  if (o.field_emission && !o.electrons_per_macroparticle)
    return serr(SPIFFE_ERR_INVALID, "specify electrons_per_macroparticle with field_emission");
  if (o.field_emission && !o.work_function)
    return serr(SPIFFE_ERR_INVALID, "specify work_function with field_emission");
  if (o.temperature < 0)
    return serr(SPIFFE_ERR_INVALID, "temperature should be a positive quantity");
  if (o.temperature > 0 && o.work_function > 0 && o.distribution_correction_interval)
    return serr(SPIFFE_ERR_INVALID, "can't do distribution correction with Richardson-Schottky emission model");
  if (add_thermal && !(o.temperature > 0 || determine_temperature))
    return serr(SPIFFE_ERR_INVALID, "add_thermal_velocities is nonzero but the temperature is not positive");
  if (add_thermal)
    return serr(SPIFFE_ERR_UNSUPPORTED, "define_cathode: add_thermal_velocities is not supported");
  if (halton_dt || halton_r)
    return serr(SPIFFE_ERR_UNSUPPORTED, "define_cathode: Halton sequences are not supported");
  if (o.random_number_seed == 0)
    return serr(SPIFFE_ERR_UNSUPPORTED, "define_cathode: a clock-generated random_number_seed (0) is not supported");
  if (determine_temperature) {
    // cathode.c:134-147, Richardson-Dushman solved for T by iteration
    if (o.work_function <= 0 || o.current_density <= 0)
      return serr(SPIFFE_ERR_INVALID, "to determine temperature, must have positive work function and current density");
    double last = 1273, t = last;
    for (int i = 0; i < 100; i++) {
      t = -SPIFFE_E_MKS * o.work_function / SPIFFE_KB_MKS / std::log(o.current_density / 60e4 / (last * last));
      if (std::fabs(last - t) < 0.01)
        break;
      last = t;
    }
    o.temperature = t;
    say("Temperature determined to be %f K\n", t);
  }
  SessionCathode c;
  if (have_profile) {
    if (tname.empty() || fname.empty())
      return serr(SPIFFE_ERR_INVALID, "define_cathode: profile needs profile_time_name and profile_factor_name");
    std::vector<std::vector<double>> cols;
    std::string err;
    if (!spiffe_sdds::read_columns(profile, {tname, fname}, cols, err))
      return serr(SPIFFE_ERR_INVALID, "define_cathode: %s", err.c_str());
    if (cols[0].empty())
      return serr(SPIFFE_ERR_INVALID, "no data in profile file");
    c.t = cols[0];
    c.A = cols[1];
    o.n_profile = (int32_t)c.t.size();
    o.profile_t = c.t.data();
    o.profile_A = c.A.data();
  }
  S_TRY(spiffe_cathode_check(&mesh, &o));
  o.profile_t = o.profile_A = nullptr;
  c.o = o;
  cathodes.push_back(std::move(c));
  return 0;
}

// ------------------------------------------------------ define_field_sampling

// the component and direction names of field_sampling.c:28-44 (units of the
// single-component columns)
static const std::vector<std::string> SAMPLE_NAMES = {"Ez", "Er", "Ephi", "Bz", "Br", "Bphi",
                                                      "Jz", "Jr", "Phi", "Q", "EAll", "BAll"};
static const char *SAMPLE_UNITS[10] = {"V/m", "V/m", "V/m", "T", "T", "T", "A/m$a2$n", "A/m$a2$n", "V", "C"};

// process_sampling_definition, field_sampling.c:53-101
int spiffe_session::cmd_field_sampling(Args &g)
{
  std::string filename, component, direction;
  spiffe_sample_options o{};
  const bool have_file = g.str("filename", filename);
  const bool have_comp = g.str("component", component);
  const bool have_dir = g.str("direction", direction);
  long long seq = 0;
  g.num("min_coord", o.min_coord);
  g.num("max_coord", o.max_coord);
  g.num("position", o.position);
  g.num("time_interval", o.time_interval);
  g.num("start_time", o.start_time);
  g.integer("time_sequence", seq);
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "you must defined the problem geometry before specifying field sampling");
  if (!have_file)
    return serr(SPIFFE_ERR_INVALID, "no filename given for field samples");
  if (!have_comp)
    return serr(SPIFFE_ERR_INVALID, "no field component named for field samples");
  if ((o.component = match(component, SAMPLE_NAMES)) < 0)
    return serr(SPIFFE_ERR_INVALID, "field component name is not recognized");
  if (o.component == SPIFFE_SAMPLE_EPHI || o.component == SPIFFE_SAMPLE_BPHI || o.component == SPIFFE_SAMPLE_BZ) {
    if (!(mesh.modes & SPIFFE_FL_TE_FIELDS))
      return serr(SPIFFE_ERR_INVALID, "can't sample TE fields unless they are enabled in define_geometry namelist");
  } else if (!(mesh.modes & SPIFFE_FL_TM_FIELDS)) {
    return serr(SPIFFE_ERR_INVALID, "can't sample TM fields/potential unless they are enabled in define_geometry namelist");
  }
  if (!have_dir)
    return serr(SPIFFE_ERR_INVALID, "no direction named for field samples");
  if ((o.direction = match(direction, {"z", "r"})) < 0)
    return serr(SPIFFE_ERR_INVALID, "direction name is not recognized");
  if (o.min_coord > o.max_coord)
    return serr(SPIFFE_ERR_INVALID, "min_coord > max_coord for field samples");
  if (o.time_interval <= 0)
    return serr(SPIFFE_ERR_INVALID, "time_interval <=0 for field samples");
  o.time_sequence = (int32_t)seq;
  SessionSampling d;
  d.o = o;
  d.path = compose(filename, rootname);
  samplings.push_back(std::move(d));
  return 0;
}

// The samples since the last flush, written as sample_fields writes them:
// a page per sample (z or r, then the component columns; rSample or zSample
// fixed, runName, tSample per page), or for a time sequence one page of rows
// (t and the component columns) rewritten with the rows so far.
int spiffe_session::flush_samples()
{
  using namespace spiffe_sdds;
  for (SessionSampling &d : samplings) {
    if (d.index < 0)
      continue;
    spiffe_sample_set h{};
    S_TRY(spiffe_gpu_download_samples(inst, d.index, &h));
    if (!h.n_samples)
      continue;
    const int64_t ns = h.n_samples, nr = h.n_rows;
    std::vector<double> t((size_t)ns), param(3 * (size_t)ns), x((size_t)nr), v[3];
    std::vector<int64_t> rows((size_t)ns);
    const int c = d.o.component, ncol = c == SPIFFE_SAMPLE_E || c == SPIFFE_SAMPLE_B ? 3 : 1;
    for (int q = 0; q < ncol; q++)
      v[q].resize((size_t)nr);
    h.max_samples = ns;
    h.max_rows = nr;
    h.t = t.data();
    h.param = param.data();
    h.rows = rows.data();
    h.x = x.data();
    for (int q = 0; q < ncol; q++)
      h.v[q] = v[q].data();
    S_TRY(spiffe_gpu_download_samples(inst, d.index, &h));
    // column names: the component, or its three (field_sampling.c:179-203)
    std::vector<Def> cols;
    const bool zdir = d.o.direction == 0, seq = d.o.time_sequence != 0;
    cols.push_back(seq ? Def{"t", "s", "", T_DOUBLE} : Def{zdir ? "z" : "r", "m", "", T_DOUBLE});
    if (ncol == 3) {
      const int base = c == SPIFFE_SAMPLE_E ? 0 : 3;
      for (int q = 0; q < 3; q++)
        cols.push_back(Def{SAMPLE_NAMES[(size_t)(base + q)], SAMPLE_UNITS[base + q], "", T_DOUBLE});
    } else {
      cols.push_back(Def{SAMPLE_NAMES[(size_t)c], SAMPLE_UNITS[c], "", T_DOUBLE});
    }
    auto fixed = [](const char *name, const char *units, const char *fmt, double value) {
      Def p{name, units, "", T_DOUBLE};
      char buf[64];
      snprintf(buf, sizeof(buf), fmt, value);
      p.fixed = true;
      p.fixed_value = buf;
      return p;
    };
    Def run{"runName", "", "", T_STRING};
    run.fixed = true;
    run.fixed_value = run_name;
    std::string err;
    if (!seq) {
      if (!d.opened) {
        // the parameter values come back parsed from the same text, so they print the same
        std::vector<Def> params = {fixed(zdir ? "rSample" : "zSample", "m", "%21.15e", param[0]), run,
                                   Def{"tSample", "s", "", T_DOUBLE}};
        if (!d.out.open(d.path, "", "", params, cols, err))
          return serr(SPIFFE_ERR_INVALID, "define_field_sampling: %s", err.c_str());
        d.opened = true;
      }
      int64_t r = 0;
      for (int64_t k = 0; k < ns; k++) {
        std::vector<const void *> cp = {x.data() + r};
        for (int q = 0; q < ncol; q++)
          cp.push_back(v[q].data() + r);
        if (!d.out.write_page({t[(size_t)k]}, {}, rows[(size_t)k], cp, err))
          return serr(SPIFFE_ERR_INVALID, "define_field_sampling: %s", err.c_str());
        r += rows[(size_t)k];
      }
    } else {
      if (d.seq_t.empty())
        std::copy(param.begin(), param.begin() + 3, d.seq_param);
      d.seq_t.insert(d.seq_t.end(), x.begin(), x.end());
      for (int q = 0; q < ncol; q++)
        d.seq_v[q].insert(d.seq_v[q].end(), v[q].begin(), v[q].end());
      Def dir{"scanDirection", "", "", T_STRING};
      dir.fixed = true;
      dir.fixed_value = zdir ? "z" : "r";
      std::vector<Def> params = {run, dir, fixed(zdir ? "rSample" : "zSample", "m", "%e", d.seq_param[0]),
                                 fixed(zdir ? "zStart" : "rStart", "m", "%e", d.seq_param[1]),
                                 fixed(zdir ? "zStop" : "rStop", "m", "%e", d.seq_param[2])};
      Writer w; // the whole page again, as the reference's updated page reads at the end
      if (!w.open(d.path, "", "", params, cols, err))
        return serr(SPIFFE_ERR_INVALID, "define_field_sampling: %s", err.c_str());
      std::vector<const void *> cp = {d.seq_t.data()};
      for (int q = 0; q < ncol; q++)
        cp.push_back(d.seq_v[q].data());
      if (!w.write_page({}, {}, (int64_t)d.seq_t.size(), cp, err))
        return serr(SPIFFE_ERR_INVALID, "define_field_sampling: %s", err.c_str());
      w.close();
    }
  }
  return 0;
}

// ------------------------------------------------------------- define_emitter

// process_emitter_definition, emitter.c:19-167; the surface is
// getBoundaryPoints' (spiffe_geometry_boundary_points)
int spiffe_session::cmd_emitter(Args &g)
{
  spiffe_emitter_options o{};
  long long material_id = -1, determine_temperature = 0, add_thermal = 0, field_emission = 0;
  long long halton_dt = 0, halton_r = 0, halton_z = 0, seed = 987654321;
  double number_per_step = 0;
  o.field_emission_beta = 1;
  o.offset_factor = 1e-2;
  std::string profile, tname, fname, log;
  g.integer("material_id", material_id);
  g.num("current_density", o.current_density);
  g.num("temperature", o.temperature);
  g.integer("determine_temperature", determine_temperature);
  g.num("work_function", o.work_function);
  g.integer("add_thermal_velocities", add_thermal);
  g.integer("field_emission", field_emission);
  g.num("field_emission_beta", o.field_emission_beta);
  g.num("electrons_per_macroparticle", o.electrons_per_macroparticle);
  g.num("start_time", o.start_time);
  g.num("stop_time", o.stop_time);
  g.num("number_per_step", number_per_step); // declared by emitter.nl, read by no code
  g.num("initial_p", o.initial_p);
  g.num("offset_factor", o.offset_factor);
  g.integer("random_number_seed", seed);
  g.integer("halton_radix_dt", halton_dt);
  g.integer("halton_radix_r", halton_r);
  g.integer("halton_radix_z", halton_z);
  const bool have_profile = g.str("profile", profile);
  g.str("profile_time_name", tname);
  g.str("profile_factor_name", fname);
  if (g.str("emission_log", log))
    warn("define_emitter: emission_log is not written");
  S_TRY(g.finish());
  o.field_emission = (int32_t)field_emission;
  if (!field_emission && o.current_density <= 0 && o.electrons_per_macroparticle == 0 && o.temperature <= 0)
    return serr(SPIFFE_ERR_INVALID,
                "either field_emission, current_density, electrons_per_macroparticle, or temperature must be non-zero");
  if (field_emission && (determine_temperature || o.current_density || have_profile))
    return serr(SPIFFE_ERR_INVALID, "field_emission is incompatible with determine_temperature, current_density, and profile");
  if (field_emission && !o.electrons_per_macroparticle)
    return serr(SPIFFE_ERR_INVALID, "specify electrons_per_macroparticle with field_emission");
  if (field_emission && !o.work_function)
    return serr(SPIFFE_ERR_INVALID, "specify work_function with field_emission");
  if (o.current_density < 0)
    return serr(SPIFFE_ERR_INVALID, "the current density should be a positive quantity");
  if (o.electrons_per_macroparticle < 0)
    return serr(SPIFFE_ERR_INVALID, "electrons_per_macroparticle should be a positive quantity");
  if (o.temperature < 0)
    return serr(SPIFFE_ERR_INVALID, "temperature should be a positive quantity");
  if (o.stop_time && o.start_time > o.stop_time)
    return serr(SPIFFE_ERR_INVALID, "stop_time is non-zero and less than start_time");
  if (add_thermal && !(o.temperature > 0 || determine_temperature))
    return serr(SPIFFE_ERR_INVALID, "add_thermal_velocities is nonzero but the temperature is not positive");
  if (add_thermal)
    return serr(SPIFFE_ERR_UNSUPPORTED, "define_emitter: add_thermal_velocities is not supported");
  if (halton_dt || halton_r || halton_z)
    return serr(SPIFFE_ERR_UNSUPPORTED, "define_emitter: Halton sequences are not supported");
  if (seed == 0)
    return serr(SPIFFE_ERR_UNSUPPORTED, "define_emitter: a clock-generated random_number_seed (0) is not supported");
  o.random_number_seed = (int32_t)seed;
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "define_emitter before define_geometry: No surface elements found");
  SessionEmitter e;
  int64_t n = 0;
  S_TRY(spiffe_geometry_boundary_points(&geo_opts, geo_text.c_str(), (int32_t)material_id, 0, nullptr, nullptr,
                                        nullptr, &n));
  if (n == 0)
    return serr(SPIFFE_ERR_INVALID, "No surface elements found with the specified material ID");
  e.iz.resize((size_t)n);
  e.ir.resize((size_t)n);
  e.dir.resize((size_t)n);
  S_TRY(spiffe_geometry_boundary_points(&geo_opts, geo_text.c_str(), (int32_t)material_id, n, e.iz.data(),
                                        e.ir.data(), e.dir.data(), &n));
  o.material_id = (int32_t)material_id;
  if (o.electrons_per_macroparticle == 0)
    return serr(SPIFFE_ERR_INVALID, "electrons_per_macroparticle must be nonzero");
  if (determine_temperature) {
    // emitter.c:98-113, Richardson-Dushman solved for T by iteration
    if (o.work_function <= 0 || o.current_density <= 0)
      return serr(SPIFFE_ERR_INVALID, "to determine temperature, must have positive work function and current density");
    double last = 1273, t = last;
    for (int i = 0; i < 100; i++) {
      t = -SPIFFE_E_MKS * o.work_function / SPIFFE_KB_MKS / std::log(o.current_density / 60e4 / (last * last));
      if (std::fabs(last - t) < 0.01)
        break;
      last = t;
    }
    o.temperature = t;
    say("Temperature determined to be %f K\n", t);
  }
  if (have_profile) {
    std::vector<std::vector<double>> cols;
    std::string err;
    if (!spiffe_sdds::read_columns(profile, {tname, fname}, cols, err))
      return serr(SPIFFE_ERR_INVALID, "define_emitter: %s", err.c_str());
    if (cols[0].empty())
      return serr(SPIFFE_ERR_INVALID, "no data in profile file");
    for (size_t i = 1; i < cols[0].size(); i++)
      if (cols[0][i - 1] >= cols[0][i])
        return serr(SPIFFE_ERR_INVALID, "profile data is not ordered by increasing time values");
    e.t = cols[0];
    e.A = cols[1];
  }
  e.o = o;
  emitters.push_back(std::move(e));
  return 0;
}

// --------------------------------------------------------- add_on_axis_fields

// process_on_axis_field_definition, onAxisFields.c:18-172
int spiffe_session::cmd_on_axis_fields(Args &g)
{
  std::string filename, z_name, Ez_name, fields_used;
  SessionOnAxis d;
  g.str("filename", filename);
  g.str("z_name", z_name);
  g.str("ez_name", Ez_name);
  g.num("ez_peak", d.Ez_peak);
  g.num("frequency", d.frequency);
  g.num("phase", d.phase);
  g.num("z_offset", d.z_offset);
  g.integer("expansion_order", d.order);
  g.str("fields_used", fields_used);
  S_TRY(g.finish());
  if (filename.empty())
    return serr(SPIFFE_ERR_INVALID, "filename is blank");
  if (z_name.empty())
    return serr(SPIFFE_ERR_INVALID, "z_name is blank");
  if (Ez_name.empty())
    return serr(SPIFFE_ERR_INVALID, "Ez_name is blank");
  if (d.Ez_peak == 0) {
    warn("Ez_peak=0, so this field is ignored.");
    return 0;
  }
  if (d.frequency == 0)
    warn("frequency=0!");
  std::vector<std::vector<double>> cols;
  std::string err;
  if (!spiffe_sdds::read_columns(filename, {z_name, Ez_name}, cols, err))
    return serr(SPIFFE_ERR_INVALID, "add_on_axis_fields: %s", err.c_str());
  d.z = cols[0];
  d.Ez = cols[1];
  OnAxisProfile p;
  d.phase = d.phase * SPIFFE_PI / 180.0; // onAxisFields.c:70
  err = onaxis_prepare(p, d.z.data(), d.Ez.data(), (int64_t)d.z.size(), d.z_offset, d.Ez_peak, d.frequency, d.phase,
                       d.order);
  if (!err.empty())
    return serr(SPIFFE_ERR_INVALID, "%s", err.c_str());
  if (onaxis.size() >= SPIFFE_MAX_ON_AXIS)
    return serr(SPIFFE_ERR_UNSUPPORTED, "more than %d on-axis fields", SPIFFE_MAX_ON_AXIS);
  onaxis.push_back(std::move(d));
  onaxis_prepared.push_back(std::move(p));
  if (fields_used.empty())
    return 0;
  // the fields of every definition so far near the axis, sine and cosine 1
  // (onAxisFields.c:130-170)
  using namespace spiffe_sdds;
  const long long nz = mesh.nz;
  std::vector<double> zc, ez, er, bp;
  for (long long iz = 0; iz < nz; iz++) {
    double Ez = 0, Er = 0, Bphi = 0;
    const double z = mesh.zmin + iz * mesh.dz;
    onaxis_eval(onaxis_prepared, z, 1e-6, 0.0, true, Ez, Er, Bphi);
    zc.push_back(z);
    ez.push_back(Ez);
    er.push_back(Er / 1e-6);
    bp.push_back(Bphi / 1e-6);
  }
  Writer w;
  if (!w.open(compose(fields_used, rootname), "", "", {},
              {Def{"z", "m", "", T_DOUBLE}, Def{"Ez", "V/m", "", T_DOUBLE}, Def{"Er/r", "V/m$a2$n", "", T_DOUBLE},
               Def{"Bphi/r", "T/m", "", T_DOUBLE}},
              err) ||
      !w.write_page({}, {}, nz, {zc.data(), ez.data(), er.data(), bp.data()}, err))
    return serr(SPIFFE_ERR_INVALID, "add_on_axis_fields: %s", err.c_str());
  return 0;
}

// ------------------------------------------------------------------ translate

// setup_translation, translate.c:21-38
int spiffe_session::cmd_translate(Args &g)
{
  if (inst)
    S_TRY(spiffe_gpu_get_mesh(inst, &mesh));
  const spiffe_mesh &m = mesh;
  double trig = m.zmax - 5 * m.dz, lower = m.zmin, upper = m.zmax;
  g.num("z_trigger", trig);
  g.num("z_lower", lower);
  g.num("z_upper", upper);
  S_TRY(g.finish());
  if (trig < m.zmin + m.dz || trig > m.zmax - m.dz)
    return serr(SPIFFE_ERR_INVALID, "z_trigger is not in range [zmin+dz, zmax-dz]");
  if (lower != upper && !(lower <= m.zmin && upper >= m.zmax))
    return serr(SPIFFE_ERR_UNSUPPORTED, "translate: reducing the integration region (z_lower, z_upper) is not supported");
  translate_on = true;
  z_trigger = trig;
  translate_set = false;
  if (inst) {
    S_TRY(spiffe_gpu_set_translation(inst, 1, z_trigger));
    translate_set = true;
  }
  return 0;
}

// ------------------------------------------------------------- define_antenna

// process_antenna_definition, antenna.c:18-107
int spiffe_session::cmd_antenna(Args &g)
{
  double start = 0, end = 0, position = 0, current = 0, frequency = 0, phase = 0, time_offset = 0;
  std::string direction = "z", waveform;
  g.num("start", start);
  g.num("end", end);
  g.num("position", position);
  g.str("direction", direction);
  g.num("current", current);
  g.num("frequency", frequency);
  g.num("phase", phase);
  const bool have_wf = g.str("waveform", waveform);
  g.num("time_offset", time_offset);
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "define_antenna before define_geometry");
  if (inst)
    S_TRY(spiffe_gpu_get_mesh(inst, &mesh));
  if (start >= end)
    return serr(SPIFFE_ERR_INVALID, "start >= end for antenna ");
  const spiffe_mesh &m = mesh;
  SessionAntenna an;
  if (direction.compare(0, 1, "r") == 0) {
    if (start < 0 || end > m.rmax)
      return serr(SPIFFE_ERR_INVALID, "antenna start or end out of range");
    if (position < m.zmin || position > m.zmax)
      return serr(SPIFFE_ERR_INVALID, "antenna position out of range");
    an.istart = (long)(start / m.dr + 0.5);
    an.iend = (long)(end / m.dr + 0.5);
    an.iposition = (long)((position - m.zmin) / m.dz);
    an.direction = 1;
  } else if (direction.compare(0, 3, "phi") == 0) {
    if (start < m.zmin || end > m.zmax)
      return serr(SPIFFE_ERR_INVALID, "antenna start or end out of range");
    if (position < 0 || position > m.rmax)
      return serr(SPIFFE_ERR_INVALID, "antenna position out of range");
    an.istart = (long)((start - m.zmin) / m.dz);
    an.iend = (long)((end - m.zmin) / m.dz);
    an.iposition = (long)(position / m.dr);
    an.direction = 2;
  } else if (direction.empty() || direction.compare(0, 1, "z") == 0) {
    if (start < m.zmin || end > m.zmax)
      return serr(SPIFFE_ERR_INVALID, "antenna start or end out of range");
    if (position < 0 || position > m.rmax)
      return serr(SPIFFE_ERR_INVALID, "antenna position out of range");
    an.istart = (long)((start - m.zmin) / m.dz + 0.5);
    an.iend = (long)((end - m.zmin) / m.dz + 0.5);
    an.iposition = (long)(position / m.dr);
    an.direction = 0;
  } else {
    return serr(SPIFFE_ERR_INVALID, "unknown antenna direction %s", direction.c_str());
  }
  if (!(an.current = current))
    warn("zero current antenna will be ignored");
  if ((an.frequency = frequency) <= 0)
    return serr(SPIFFE_ERR_INVALID, "antenna frequency <= 0");
  an.phase = phase;
  if (!have_wf)
    return serr(SPIFFE_ERR_INVALID, "no antenna waveform file given");
  std::vector<std::vector<double>> cols;
  std::string err;
  if (!spiffe_sdds::read_columns(waveform, {"t", "W"}, cols, err))
    return serr(SPIFFE_ERR_INVALID, "define_antenna: %s", err.c_str());
  if (cols[0].size() <= 2)
    return serr(SPIFFE_ERR_INVALID, "SDDS waveform file empty or invalid");
  an.t = cols[0];
  an.W = cols[1];
  for (double &t : an.t)
    t += time_offset;
  for (size_t i = 1; i < an.t.size(); i++)
    if (an.t[i - 1] >= an.t[i])
      return serr(SPIFFE_ERR_INVALID, "waveform data is not ordered by increasing time index");
  antennas.push_back(std::move(an));
  return 0;
}

// --------------------------------------------------------------- define_screen

// process_screen_definition, screens.c:29-117
// processSecondaryEmissionDefinition, secondaryEmission.c:21-118
int spiffe_session::cmd_secondary_emission(Args &g)
{
  std::string input_file, energy_col, yield_col, log_file;
  double yield_limit = 0, emitted_momentum = 0;
  long long verbosity = 1, material_id = 1;
  const bool have_input = g.str("input_file", input_file);
  const bool have_energy = g.str("kinetic_energy_column", energy_col);
  const bool have_yield = g.str("yield_column", yield_col);
  g.num("yield_limit", yield_limit);
  g.num("emitted_momentum", emitted_momentum);
  g.integer("verbosity", verbosity);
  g.integer("material_id", material_id);
  const bool have_log = g.str("log_file", log_file);
  S_TRY(g.finish());
  if (!have_input || input_file.empty())
    return serr(SPIFFE_ERR_INVALID, "supply an input file");
  if (!have_energy || energy_col.empty())
    return serr(SPIFFE_ERR_INVALID, "supply the name of a column containing energy values");
  if (!have_yield || yield_col.empty())
    return serr(SPIFFE_ERR_INVALID, "supply the name of a column containing yield values");
  if (emitted_momentum < 0)
    return serr(SPIFFE_ERR_INVALID, "emitted_momentum < 0");
  std::vector<std::vector<double>> cols;
  std::string err;
  if (!spiffe_sdds::read_columns(input_file, {energy_col, yield_col}, cols, err))
    return serr(SPIFFE_ERR_INVALID, "problem reading secondary emission yield data file: %s", err.c_str());
  if (cols[0].empty())
    return serr(SPIFFE_ERR_INVALID, "no data in yield file");
  SessionSecondary d;
  d.o.material_id = (int32_t)material_id;
  d.o.verbosity = (int32_t)verbosity;
  d.o.emitted_momentum = emitted_momentum;
  d.o.yield_limit = (int64_t)yield_limit;
  d.E = cols[0];
  d.Y = cols[1];
  for (size_t i = 1; i < d.E.size(); i++)
    if (d.E[i - 1] >= d.E[i])
      return serr(SPIFFE_ERR_INVALID, "secondary emission data is not ordered by increasing energy values");
  if (have_log && !log_file.empty()) { // :91-114
    using namespace spiffe_sdds;
    const std::vector<Def> lc = {Def{"z", "m", "", T_FLOAT},      Def{"r", "m", "", T_FLOAT},
                                 Def{"t", "s", "", T_FLOAT},      Def{"K", "eV", "", T_FLOAT},
                                 Def{"yield", "", "", T_FLOAT},   Def{"emitted", "", "", T_SHORT},
                                 Def{"directionCode", "", "", T_SHORT}, Def{"generation", "", "", T_SHORT},
                                 Def{"particleID", "", "", T_LONG}};
    if (!d.log_out.open(compose(log_file, rootname), "Primary/secondary activity due to material " + input_file,
                        "", {}, lc, err))
      return serr(SPIFFE_ERR_INVALID, "define_secondary_emission log_file: %s", err.c_str());
    d.o.log = 1;
  }
  secondaries.push_back(std::move(d));
  return 0;
}

// The secondary-emission log pages since the last flush: one page per
// definition and emitting step (secondaryEmission.c:548-563).  The particleID
// column holds the IDs the log took (:541); the reference hands the short
// generation buffer to that long column (:557), which reads past its values.
int spiffe_session::flush_secondary_logs()
{
  for (size_t k = 0; k < secondaries.size(); k++) {
    SessionSecondary &d = secondaries[k];
    if (!d.log_out.is_open() || !d.on_device)
      continue;
    int64_t n = 0;
    S_TRY(spiffe_gpu_secondary_log(inst, (int32_t)k, 0, nullptr, &n));
    if (!n)
      continue;
    std::vector<double> rows((size_t)n * SPIFFE_SECONDARY_LOG_COLS);
    S_TRY(spiffe_gpu_secondary_log(inst, (int32_t)k, n, rows.data(), &n));
    const size_t C = SPIFFE_SECONDARY_LOG_COLS;
    for (size_t a = 0; a < (size_t)n;) {
      size_t b = a;
      while (b < (size_t)n && rows[b * C] == rows[a * C])
        b++;
      const size_t m = b - a;
      std::vector<float> f[5];
      std::vector<int16_t> h[3];
      std::vector<int32_t> id(m);
      for (size_t i = 0; i < m; i++) {
        const double *r = &rows[(a + i) * C];
        for (int c = 0; c < 5; c++)
          f[c].push_back((float)r[1 + c]);
        for (int c = 0; c < 3; c++)
          h[c].push_back((int16_t)r[6 + c]);
        id[i] = (int32_t)r[9];
      }
      std::vector<const void *> cols;
      for (int c = 0; c < 5; c++)
        cols.push_back(f[c].data());
      for (int c = 0; c < 3; c++)
        cols.push_back(h[c].data());
      cols.push_back(id.data());
      std::string err;
      if (!d.log_out.write_page({}, {}, (int64_t)m, cols, err))
        return serr(SPIFFE_ERR_INVALID, "define_secondary_emission log_file: %s", err.c_str());
      a = b;
    }
  }
  return 0;
}

int spiffe_session::cmd_screen(Args &g)
{
  std::string filename, templ, direction = "forward";
  double z_position = 0, delta_z = 0, start_time = 0;
  long long number = 1;
  const bool have_file = g.str("filename", filename);
  const bool have_templ = g.str("template", templ);
  g.num("z_position", z_position);
  g.num("delta_z", delta_z);
  g.integer("number_of_screens", number);
  g.num("start_time", start_time); // stored by the reference, read by no code
  g.str("direction", direction);
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "define_screen before define_geometry");
  if (number < 1)
    return serr(SPIFFE_ERR_INVALID, "number_of_screens is invalid");
  if (!have_file && number == 1)
    return serr(SPIFFE_ERR_INVALID, "no filename given for screen");
  if (!have_templ && number > 1)
    return serr(SPIFFE_ERR_INVALID, "no template given for screens");
  if (have_file && have_templ)
    return serr(SPIFFE_ERR_INVALID, "both filename and template are given--this doesn't make sense");
  const int d = match(direction, {"forward", "backward"});
  if (d < 0)
    return serr(SPIFFE_ERR_INVALID, "unknown screen direction specified");
  const char *dname = d == 0 ? "forward" : "backward";
  for (long long i = 0; i < number; i++) {
    if (screens.size() >= SPIFFE_MAX_SCREENS)
      return serr(SPIFFE_ERR_INVALID, "at most %d screens", SPIFFE_MAX_SCREENS);
    screens.emplace_back();
    SessionScreen &sc = screens.back();
    if (have_file) {
      sc.filename = compose(filename, rootname);
    } else {
      char name[1024];
      std::snprintf(name, sizeof(name), compose(templ, rootname).c_str(), (long)i);
      sc.filename = name;
    }
    sc.z = z_position;
    sc.direction = d == 0 ? 1 : -1;
    // screens.c:79-100: the reference's columns, units and parameters
    using namespace spiffe_sdds;
    std::vector<Def> cols;
    const char *q[8] = {"r", "pz", "pr", "pphi", "t", "q", "r0", "t0"};
    const char *u[8] = {"m", "m$be$nc", "m$be$nc", "m$be$nc", "s", "C", "m", "s"};
    for (int k = 0; k < 8; k++)
      cols.push_back(Def{q[k], u[k], "", T_DOUBLE});
    cols.push_back(Def{"generation", "", "", T_SHORT});
    cols.push_back(Def{"particleID", "", "", T_LONG});
    for (const char *n : {"rMin", "rMax", "zMin", "zMax"})
      cols.push_back(Def{n, "m", "", T_DOUBLE});
    std::vector<Def> params;
    Def dir{"direction", "", "", T_STRING};
    dir.fixed = true;
    dir.fixed_value = dname;
    params.push_back(dir);
    params.push_back(Def{"Time", "s", "Time of output", T_DOUBLE});
    params.push_back(Def{"Timestep", "", "Time-step of output", T_LONG});
    char label[512];
    std::snprintf(label, sizeof(label), "spiffe screen output for run %s for particles %s-crossing z=%e m",
                  rootname.c_str(), dname, z_position);
    std::string err;
    if (!sc.out.open(sc.filename, label, "", params, cols, err))
      return serr(SPIFFE_ERR_INVALID, "define_screen: %s", err.c_str());
    z_position += delta_z;
  }
  return 0;
}

// process_testbeam_definition, test_beam.c:17-56, and spiffe.c:262-268
int spiffe_session::cmd_test_beam(Args &g)
{
  spiffe_test_beam_options o{};
  double zf = 0, rf = 0, zd = DBL_MAX, rd = DBL_MAX;
  g.num("start_time", o.start_time);
  g.num("stop_time", o.stop_time);
  g.num("initial_z", o.initial_z);
  g.num("initial_r", o.initial_r);
  g.num("initial_pz", o.initial_pz);
  g.num("initial_pr", o.initial_pr);
  g.num("initial_rpphi", o.initial_rpphi);
  g.num("z_force", zf);
  g.num("r_force", rf);
  g.num("z_start_deceleration", zd);
  g.num("r_start_deceleration", rd);
  g.num("electrons_per_macroparticle", o.electrons_per_macroparticle);
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "define_test_beam before define_geometry");
  if (o.initial_z < mesh.zmin || o.initial_z > mesh.zmax)
    return serr(SPIFFE_ERR_INVALID, "test beam initial_z is outside of simulation region");
  if (o.initial_r < 0 || o.initial_r > mesh.rmax)
    return serr(SPIFFE_ERR_INVALID, "test beam initial_r is outside of simulation region");
  if (o.start_time >= o.stop_time)
    return serr(SPIFFE_ERR_INVALID, "start_time >= stop_time for test beam");
  if (o.electrons_per_macroparticle <= 0)
    return serr(SPIFFE_ERR_INVALID, "electrons_per_macroparticle <= 0 for test beam");
  if (zf < 0)
    return serr(SPIFFE_ERR_INVALID, "z_force < 0 for test beam");
  if (test_beam)
    return serr(SPIFFE_ERR_INVALID, "test beam already defined");
  if (!cathodes.empty())
    return serr(SPIFFE_ERR_INVALID, "can't do both cathode and test beam");
  test_beam = true;
  tb = o;
  tb_z_force = zf;
  tb_r_force = rf;
  tb_z_decel = zd;
  tb_r_decel = rd;
  return 0;
}

// setup_poisson_correction, poisson_correction.c:31-71
int spiffe_session::cmd_poisson(Args &g)
{
  spiffe_poisson_options o{};
  o.accuracy = 1e-6;
  o.maximum_iterations = 1000;
  double test_charge = 0, zt = 0, rt = 0;
  std::string guess = "none";
  g.num("start_time", o.start_time);
  g.integer("step_interval", o.step_interval);
  g.num("accuracy", o.accuracy);
  g.num("error_charge_threshold", o.error_charge_threshold);
  g.integer("maximum_iterations", o.maximum_iterations);
  g.integer("verbosity", o.verbosity);
  g.num("test_charge", test_charge);
  g.num("z_test_charge", zt);
  g.num("r_test_charge", rt);
  g.str("guess_type", guess);
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "poisson_correction before define_geometry");
  if (o.start_time < 0)
    return serr(SPIFFE_ERR_INVALID, "start_time < 0 for poisson_correction");
  if (o.step_interval < 0)
    return serr(SPIFFE_ERR_INVALID, "step_interval < 0 for poisson_correction");
  if (o.accuracy <= 0)
    return serr(SPIFFE_ERR_INVALID, "accuracy <= 0 for poisson_correction");
  if (o.maximum_iterations <= 0)
    return serr(SPIFFE_ERR_INVALID, "maximum iterations <= 0 for poisson_correction");
  if (o.verbosity < 0)
    return serr(SPIFFE_ERR_INVALID, "verbosity < 0 for poisson_correction");
  if (test_charge)
    return serr(SPIFFE_ERR_UNSUPPORTED, "poisson_correction: test_charge is not supported");
  if ((o.guess_code = match(guess, {"none", "line-charge", "point-charge", "zero"})) < 0)
    return serr(SPIFFE_ERR_INVALID, "unknown guess type for poisson_correction");
  if (!(mesh.modes & SPIFFE_FL_TM_FIELDS))
    return serr(SPIFFE_ERR_INVALID, "TM fields must be enabled in order to do poisson correction");
  pc = o;
  pc_defined = true;
  return 0;
}

// ---------------------------------------------------------------- load_fields

// perform_field_loading, load_fields.c:20-282: the first page at or after
// time_threshold, scaled (Ez_peak or factor) and added into the problem's
// fields, shifted by the whole-cell offset between the two meshes.
int spiffe_session::cmd_load_fields(Args &g)
{
  std::string filename;
  double Ez_peak = 0, factor = 1, time_threshold = 0;
  long long overlay = 0; // declared by load_fields.nl; loading always adds
  const bool have_file = g.str("filename", filename);
  g.num("ez_peak", Ez_peak);
  g.num("factor", factor);
  g.num("time_threshold", time_threshold);
  g.integer("overlay", overlay);
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "load_fields before define_geometry");
  if (!have_file)
    return serr(SPIFFE_ERR_INVALID, "no filename given for field samples");
  if (Ez_peak == 0 && factor == 0)
    return serr(SPIFFE_ERR_INVALID, "Ez_peak and factor cannot both be zero");
  using namespace spiffe_sdds;
  Reader r;
  std::string err;
  if (!r.open(filename, err))
    return serr(SPIFFE_ERR_INVALID, "load_fields: %s", err.c_str());
  // checkLoadFile, load_fields.c:284-312
  const char *pnames[] = {"time", "version", "nr", "nz", "dr", "dz", "zmin", "zmax", "rmax", "zt", "TMfields",
                          "TEfields"};
  int pi[12];
  for (int k = 0; k < 12; k++)
    if ((pi[k] = r.param_index(pnames[k])) < 0)
      return serr(SPIFFE_ERR_INVALID, "load file is invalid--check presence, type, and units of data");
  if (r.column_index("metalFlags") < 0)
    return serr(SPIFFE_ERR_INVALID, "load file is invalid--check presence, type, and units of data");
  Page p;
  bool found = false;
  while (r.next_page(p, err)) {
    if (p.param[(size_t)pi[0]] < time_threshold)
      continue;
    found = true;
    break;
  }
  if (!found)
    return serr(SPIFFE_ERR_INVALID, "unable to get data for field loading%s%s", err.empty() ? "" : ": ", err.c_str());
  say("Using fields from t = %es\n", p.param[(size_t)pi[0]]);
  const long long lnr = (long long)p.param[(size_t)pi[2]], lnz = (long long)p.param[(size_t)pi[3]];
  const double lzmin = p.param[(size_t)pi[6]], lzmax = p.param[(size_t)pi[7]], lrmax = p.param[(size_t)pi[8]];
  const bool tm = p.param_text[(size_t)pi[10]] == "y", te = p.param_text[(size_t)pi[11]] == "y";
  const int64_t rows = (lnz + 1) * (lnr + 1);
  if (p.rows != rows)
    return serr(SPIFFE_ERR_INVALID, "load_fields: page holds %lld rows, nz and nr give %lld", (long long)p.rows,
                (long long)rows);
  const char *tmn[6] = {"Ez", "Er", "Jz", "Jr", "Bphi", "Bphi2"};
  const char *ten[6] = {"Ephi", "Jphi", "Br", "Br2", "Bz", "Bz2"};
  std::map<std::string, std::vector<double> *> L;
  auto take = [&](const char *n) -> bool {
    const int c = r.column_index(n);
    if (c < 0 || p.col[(size_t)c].size() != (size_t)rows)
      return false;
    L[n] = &p.col[(size_t)c];
    return true;
  };
  if (tm)
    for (const char *n : tmn)
      if (!take(n))
        return serr(SPIFFE_ERR_INVALID, "unable to get TM field columns as matrices");
  if (te)
    for (const char *n : ten)
      if (!take(n))
        return serr(SPIFFE_ERR_INVALID, "unable to get TE field columns as matrices");
  const long long P = lnr + 1;
  if (Ez_peak) {
    if (!tm)
      return serr(SPIFFE_ERR_INVALID, "can't scale Ez_peak because TM mode fields are not enabled");
    const std::vector<double> &Ez = *L["Ez"];
    double Ez_max = 0, z_max = 0;
    for (long long iz = 1; iz <= lnz; iz++)
      if (std::fabs(Ez_max) < std::fabs(Ez[(size_t)(iz * P)])) {
        Ez_max = Ez[(size_t)(iz * P)];
        z_max = (iz - 0.5) * p.param[(size_t)pi[5]] + lzmin;
      }
    if (std::fabs(Ez_max) < 1e-10)
      return serr(SPIFFE_ERR_INVALID, "extremal value of on-axis Ez is < 1e-10--can't scale up");
    say("Extremal value of on-axis Ez is %e V at z = %e m.\n", Ez_max, z_max);
    factor = Ez_peak / Ez_max;
  }
  if (factor != 1)
    for (auto &kv : L)
      for (double &v : *kv.second)
        v *= factor;
  // the overlay, load_fields.c:173-242
  S_TRY(pull());
  const spiffe_mesh &m = mesh;
  long long iz_start = 0, iz_end = m.nz, iz_offset = 0, ir_end = m.nr;
  const double dz1 = (m.zmax - m.zmin) / (m.nz - 1), dz = (lzmax - lzmin) / (lnz - 1);
  const double dr1 = m.rmax / (m.nr - 1), dr = lrmax / (lnr - 1);
  if (lnz != m.nz || lnr != m.nr || lzmax != m.zmax || lzmin != m.zmin || lrmax != m.rmax) {
    warn("possible geometry mismatch in overlay fields");
    if (std::fabs(dz / dz1 - 1) > 1e-6)
      return serr(SPIFFE_ERR_INVALID, "dz's not close enough");
    if (std::fabs(dr / dr1 - 1) > 1e-6)
      return serr(SPIFFE_ERR_INVALID, "dr's not close enough");
    iz_offset = (long long)((m.zmin - lzmin) / dz + 0.5);
    if (std::fabs(iz_offset - (m.zmin - lzmin) / dz) > 1e-6)
      return serr(SPIFFE_ERR_INVALID, "misalignment of boundary and grid lines from existing data and data in file");
    if (iz_offset < 0)
      iz_start = -iz_offset;
    if (m.nz + iz_offset > lnz)
      iz_end = lnz - iz_offset;
    // the reference sets ir_end to the larger nr here and so runs past the
    // smaller of the two meshes; the overlap is the rows both hold
    ir_end = m.nr < lnr ? m.nr : lnr;
  }
  const long long Pm = m.nr + 1;
  auto add = [&](const char *dst, const char *src) -> int {
    if (!has(dst))
      return serr(SPIFFE_ERR_INVALID, "attempt to overlay %s onto problem which does not contain it", dst);
    std::vector<double> &A = a[dst];
    const std::vector<double> &B = *L[src];
    for (long long iz = iz_start; iz <= iz_end; iz++)
      for (long long ir = 0; ir <= ir_end; ir++)
        A[(size_t)(iz * Pm + ir)] += B[(size_t)((iz + iz_offset) * P + ir)];
    return 0;
  };
  if (tm) {
    if (!(m.modes & SPIFFE_FL_TM_FIELDS))
      return serr(SPIFFE_ERR_INVALID, "attempt to overlay TM mode fields onto problem which does not contain those fields");
    for (const char *n : tmn)
      S_TRY(add(n, n));
  }
  if (te) {
    if (!(m.modes & SPIFFE_FL_TE_FIELDS))
      return serr(SPIFFE_ERR_INVALID, "attempt to overlay TE mode fields onto problem which does not contain those fields");
    for (const char *n : ten)
      S_TRY(add(n, n));
  }
  say("fields added to pre-existing problem\n");
  return push_fields({"Ez", "Er", "Jz", "Jr", "Bphi", "Bphi2", "Ephi", "Jphi", "Br", "Br2", "Bz", "Bz2"});
}

// process_field_saving_definition, field_saving.c:16-44
int spiffe_session::cmd_field_saving(Args &g)
{
  std::string filename;
  double time_interval = -1, start_time = 0, trigger = -1;
  long long save_before_exiting = 0;
  const bool have_file = g.str("filename", filename);
  g.num("time_interval", time_interval);
  g.num("start_time", start_time);
  g.integer("save_before_exiting", save_before_exiting);
  g.num("z_ez_trigger", trigger);
  S_TRY(g.finish());
  if (!have_file)
    return serr(SPIFFE_ERR_INVALID, "no filename given for field samples");
  if (trigger != -1 && time_interval != -1)
    return serr(SPIFFE_ERR_INVALID, "Either use time_interval or iz_Ez_trigger, not both");
  if (time_interval == -1 && trigger == -1)
    return serr(SPIFFE_ERR_INVALID, "Use one of time_interval or iz_Ez_trigger");
  if (trigger != -1)
    return serr(SPIFFE_ERR_UNSUPPORTED, "define_field_saving: saving on an Ez trigger is not supported");
  if (time_interval < 0)
    return serr(SPIFFE_ERR_INVALID, "define_field_saving: time_interval < 0");
  saving.out.close();
  saving.defined = true;
  saving.filename = filename;
  saving.time_interval = time_interval;
  saving.start_time = start_time;
  saving.save_before_exiting = save_before_exiting;
  saving.step_interval = saving.start_step = -1;
  saving.save_index = -1;
  return 0;
}

// save_fields, field_saving.c:46-213 (time_interval schedule)
int spiffe_session::save_fields(long long step, double time, bool final_call)
{
  if (!saving.defined)
    return 0;
  using namespace spiffe_sdds;
  const spiffe_mesh &m = mesh;
  if (saving.save_index == -1) {
    saving.step_interval = (long long)(saving.time_interval / m.dt + 0.5);
    saving.start_step = (long long)((saving.start_time - m.start_time) / m.dt + 0.5);
    saving.save_index = 0;
    auto fixed = [](const char *n, const char *u, const char *d, Type t, const std::string &v) {
      Def x{n, u, d, t};
      x.fixed = true;
      x.fixed_value = v;
      return x;
    };
    auto num = [](double v) {
      char b[64];
      std::snprintf(b, sizeof(b), "%.17g", v);
      return std::string(b);
    };
    std::vector<Def> params = {Def{"time", "s", "time of field save", T_DOUBLE},
                               fixed("version", "", "save version", T_LONG, "4"),
                               fixed("nr", "", "number of r grid lines", T_LONG, std::to_string(m.nr)),
                               fixed("nz", "", "number of z grid lines", T_LONG, std::to_string(m.nz)),
                               fixed("dr", "m", "spacing of r grid lines", T_DOUBLE, num(m.dr)),
                               fixed("dz", "m", "spacing of z grid lines", T_DOUBLE, num(m.dz)),
                               fixed("zmin", "m", "", T_DOUBLE, num(m.zmin)),
                               fixed("zmax", "m", "", T_DOUBLE, num(m.zmax)),
                               fixed("rmax", "m", "", T_DOUBLE, num(m.rmax)),
                               fixed("zt", "m", "", T_DOUBLE, num(0)),
                               fixed("TMfields", "", "", T_CHARACTER, m.modes & SPIFFE_FL_TM_FIELDS ? "y" : "n"),
                               fixed("TEfields", "", "", T_CHARACTER, m.modes & SPIFFE_FL_TE_FIELDS ? "y" : "n")};
    std::vector<Def> cols = {Def{"metalFlags", "", "", T_LONG}};
    if (m.modes & SPIFFE_FL_TM_FIELDS)
      for (auto &c : {std::make_pair("Ez", "V/m"), std::make_pair("Er", "V/m"), std::make_pair("Jz", "A/m$a2$n"),
                      std::make_pair("Jr", "A/m$a2$n"), std::make_pair("Bphi", "T"), std::make_pair("Bphi2", "T")})
        cols.push_back(Def{c.first, c.second, "", T_DOUBLE});
    if (m.modes & SPIFFE_FL_TE_FIELDS)
      for (auto &c : {std::make_pair("Ephi", "V/m"), std::make_pair("Jphi", "A/m$a2$n"), std::make_pair("Br", "T"),
                      std::make_pair("Br2", "T"), std::make_pair("Bz", "T"), std::make_pair("Bz2", "T")})
        cols.push_back(Def{c.first, c.second, "", T_DOUBLE});
    std::string err;
    if (!saving.out.open(compose(saving.filename, rootname), "", "spiffe field saves", params, cols, err))
      return serr(SPIFFE_ERR_INVALID, "field saving: %s", err.c_str());
  }
  bool save = false;
  if (final_call && saving.save_before_exiting)
    save = true;
  else
    save = due(step, saving.start_step, saving.step_interval);
  if (!save)
    return 0;
  S_TRY(pull());
  const size_t n = nodes();
  // the reference defines metalFlags but never sets it (field_saving.c:154-193)
  std::vector<int32_t> zero_flags(n, 0);
  std::vector<const void *> cols = {zero_flags.data()};
  if (m.modes & SPIFFE_FL_TM_FIELDS)
    for (const char *c : {"Ez", "Er", "Jz", "Jr", "Bphi", "Bphi2"})
      cols.push_back(a[c].data());
  if (m.modes & SPIFFE_FL_TE_FIELDS)
    for (const char *c : {"Ephi", "Jphi", "Br", "Br2", "Bz", "Bz2"})
      cols.push_back(a[c].data());
  std::string err;
  if (!saving.out.write_page({time}, {""}, (int64_t)n, cols, err))
    return serr(SPIFFE_ERR_INVALID, "field saving: %s", err.c_str());
  say("fields saved to file %s at t=%e s\n", saving.filename.c_str(), time);
  saving.save_index++;
  return 0;
}

// process_snapshot_definition, snapshots.c:16-40
int spiffe_session::cmd_snapshots(Args &g)
{
  std::string filename;
  double time_interval = 0, start_time = 0;
  const bool have_file = g.str("filename", filename);
  g.num("time_interval", time_interval);
  g.num("start_time", start_time);
  S_TRY(g.finish());
  if (!have_file)
    return serr(SPIFFE_ERR_INVALID, "no filename given for beam snapshots");
  if (time_interval < 0)
    return serr(SPIFFE_ERR_INVALID, "time_interval < 0 for beam snapshots");
  snapshots.out.close();
  snapshots.defined = true;
  snapshots.filename = compose(filename, rootname);
  snapshots.time_interval = time_interval;
  snapshots.start_time = start_time;
  snapshots.step_interval = snapshots.start_step = snapshots.index = -1;
  return 0;
}

// take_beam_snapshot, snapshots.c:48-119: the beam at the step's start
int spiffe_session::take_snapshot(long long step, double time)
{
  if (!snapshots.defined)
    return 0;
  using namespace spiffe_sdds;
  BeamSnapshots &S = snapshots;
  if (S.index == -1) {
    S.step_interval = (long long)(S.time_interval / mesh.dt + 0.5);
    S.start_step = (long long)((S.start_time - mesh.start_time) / mesh.dt + 0.5);
    S.index = 0;
    const char *q[9] = {"z", "r", "pz", "pr", "pphi", "q", "r0", "z0", "t0"};
    const char *u[9] = {"m", "m", "m$be$nc", "m$be$nc", "m$be$nc", "C", "m", "m", "s"};
    std::vector<Def> cols;
    for (int k = 0; k < 9; k++)
      cols.push_back(Def{q[k], u[k], "", T_DOUBLE});
    cols.push_back(Def{"generation", "", "", T_SHORT});
    cols.push_back(Def{"particleID", "", "", T_LONG});
    cols.push_back(Def{"status", "", "", T_SHORT});
    std::vector<Def> params = {Def{"Time", "s", "Time of snapshot", T_DOUBLE},
                               Def{"Timestep", "", "Time-step of snapshot", T_LONG}};
    std::string err;
    if (!S.out.open(S.filename, "spiffe beam snapshots for run " + rootname, "", params, cols, err))
      return serr(SPIFFE_ERR_INVALID, "beam snapshots: %s", err.c_str());
  }
  if (!due(step, S.start_step, S.step_interval))
    return 0;
  int64_t np = 0;
  S_TRY(spiffe_gpu_counts(inst, &np, nullptr));
  const size_t n = (size_t)np, cap = n ? n : 1;
  std::vector<std::vector<double>> d(16, std::vector<double>(cap));
  std::vector<int32_t> id(cap);
  std::vector<int16_t> gen(cap);
  std::vector<uint64_t> st(cap);
  spiffe_beam_set b{};
  b.capacity = (int64_t)cap;
  double **ptr[16] = {&b.z, &b.r, &b.pz, &b.pr, &b.r_pphi, &b.vz, &b.vr, &b.vphi, &b.Q, &b.r0, &b.z0, &b.t0,
                      &b.rmin, &b.rmax, &b.zmin, &b.zmax};
  for (int k = 0; k < 16; k++)
    *ptr[k] = d[(size_t)k].data();
  b.particleID = id.data();
  b.generation = gen.data();
  b.status = st.data();
  S_TRY(spiffe_gpu_download_beam(inst, &b));
  std::vector<double> pphi(cap);
  std::vector<int16_t> status(cap);
  for (size_t i = 0; i < n; i++) {
    pphi[i] = b.r[i] ? b.r_pphi[i] / b.r[i] : 0.0;
    status[i] = (int16_t)b.status[i];
  }
  std::vector<const void *> cols = {b.z, b.r, b.pz, b.pr, pphi.data(), b.Q, b.r0, b.z0, b.t0,
                                    gen.data(), id.data(), status.data()};
  std::string err;
  if (!S.out.write_page({time, (double)step}, {"", ""}, np, cols, err))
    return serr(SPIFFE_ERR_INVALID, "beam snapshots: %s", err.c_str());
  say("beam snapshot saved to file %s at t=%.16e, step %lld\n", S.filename.c_str(), time, step);
  S.index++;
  return 0;
}

// process_field_output_definition, field_output.c:16-43
int spiffe_session::cmd_field_output(Args &g)
{
  std::string filename;
  FieldOutput o;
  const bool have_file = g.str("filename", filename);
  g.num("time_interval", o.time_interval);
  g.num("start_time", o.start_time);
  g.integer("z_interval", o.z_interval);
  g.integer("r_interval", o.r_interval);
  g.integer("exclude_imposed_field", o.exclude_imposed);
  g.integer("separate_imposed_field", o.separate_imposed);
  S_TRY(g.finish());
  if (!have_file)
    return serr(SPIFFE_ERR_INVALID, "no filename given for field samples");
  if (o.time_interval < 0)
    return serr(SPIFFE_ERR_INVALID, "time_interval < 0 for field samples");
  if (o.z_interval < 1 || o.r_interval < 1)
    return serr(SPIFFE_ERR_INVALID, "z_interval and r_interval must be > 1");
  o.defined = true;
  o.filename = compose(filename, rootname);
  field_output = std::move(o);
  return 0;
}

// output_fields, field_output.c:45-214: node-centred fields every
// z_interval-th row and r_interval-th column, single precision
int spiffe_session::output_fields(long long step, double time)
{
  if (!field_output.defined)
    return 0;
  using namespace spiffe_sdds;
  FieldOutput &O = field_output;
  const spiffe_mesh &m = mesh;
  const bool tm = m.modes & SPIFFE_FL_TM_FIELDS, te = m.modes & SPIFFE_FL_TE_FIELDS;
  const bool sep = tm && O.separate_imposed;
  if (O.index == -1) {
    O.step_interval = (long long)(O.time_interval / m.dt + 0.5);
    O.start_step = (long long)((O.start_time - m.start_time) / m.dt + 0.5);
    O.index = 0;
    Def v1{"Variable1Name", "", "", T_STRING}, v2{"Variable2Name", "", "", T_STRING};
    v1.fixed = v2.fixed = true;
    v1.fixed_value = "z";
    v2.fixed_value = "r";
    std::vector<Def> params = {v1, Def{"zMinimum", "m", "", T_DOUBLE}, Def{"zInterval", "m", "", T_DOUBLE},
                               Def{"zDimension", "m", "", T_LONG}, Def{"rMinimum", "m", "", T_DOUBLE},
                               Def{"rInterval", "m", "", T_DOUBLE}, Def{"rDimension", "m", "", T_LONG}, v2,
                               Def{"Time", "s", "Time of output", T_DOUBLE},
                               Def{"Timestep", "", "Time-step of output", T_LONG}};
    std::vector<Def> cols = {Def{"z", "m", "", T_FLOAT}, Def{"r", "m", "", T_FLOAT},
                             Def{"rho", "C/m$a3$n", "", T_FLOAT}};
    if (tm) {
      for (auto &c : {std::make_pair("Ez", "V/m"), std::make_pair("Er", "V/m"), std::make_pair("Bphi", "T"),
                      std::make_pair("Jz", "A/m$a2$n"), std::make_pair("Jr", "A/m$a2$n")})
        cols.push_back(Def{c.first, c.second, "", T_FLOAT});
      if (sep) {
        cols.push_back(Def{"EzImposed", "V/m", "", T_FLOAT});
        cols.push_back(Def{"ErImposed", "V/m", "", T_FLOAT});
      }
    }
    if (te)
      for (auto &c : {std::make_pair("Ephi", "V/m"), std::make_pair("Br", "T"), std::make_pair("Bz", "T"),
                      std::make_pair("Jphi", "A/m$a2$n")})
        cols.push_back(Def{c.first, c.second, "", T_FLOAT});
    std::string err;
    if (!O.out.open(O.filename, "", "spiffe field output", params, cols, err))
      return serr(SPIFFE_ERR_INVALID, "field output: %s", err.c_str());
  }
  if (!due(step, O.start_step, O.step_interval))
    return 0;
  O.index++;
  S_TRY(pull());
  const long long nz = m.nz, nr = m.nr, P = nr + 1;
  const double dr2 = m.dr * m.dr;
  std::vector<double> area_c((size_t)nr + 1); // calculate_areas, integrate.c:689-701
  for (long long ir = 0; ir <= nr; ir++)
    area_c[(size_t)ir] = ir ? SPIFFE_PIx2 * ir * dr2 : SPIFFE_PI * dr2 / 4;
  std::vector<std::vector<float>> col(16);
  auto A = [&](const char *n) -> const double * { return has(n) ? a[n].data() : nullptr; };
  const double *Q = A("Q"), *Ez = A("Ez"), *Er = A("Er"), *Jz = A("Jz"), *Jr = A("Jr"), *B2 = A("Bphi2");
  const double *EzI = A("EzImposed"), *ErI = A("ErImposed"), *Ephi = A("Ephi"), *Jphi = A("Jphi");
  const double *Br2 = A("Br2"), *Bz2 = A("Bz2");
  for (long long iz = 0; iz < nz; iz += O.z_interval) {
    const float zv = (float)(iz * m.dz + m.zmin);
    for (long long ir = 0; ir < nr; ir += O.r_interval) {
      const size_t i = (size_t)(iz * P + ir), iu = i + (size_t)P, ir1 = i + 1;
      int c = 0;
      col[(size_t)c++].push_back(zv);
      col[(size_t)c++].push_back((float)(ir * m.dr));
      col[(size_t)c++].push_back((float)(Q[i] / (m.dz * area_c[(size_t)ir])));
      if (tm) {
        const float ezi = (float)((EzI[i] + EzI[iu]) / 2);
        const float ez = (float)((Ez[i] + Ez[iu]) / 2 + (O.exclude_imposed ? 0 : ezi));
        const float eri = (float)((ErI[i] + ErI[iu]) / 2); // as field_output.c:162, row iz+1
        const float er = (float)((Er[i] + Er[ir1]) / 2 + (O.exclude_imposed ? 0 : eri));
        col[(size_t)c++].push_back(ez);
        col[(size_t)c++].push_back(er);
        col[(size_t)c++].push_back((float)((B2[i] + B2[ir1] + B2[iu] + B2[iu + 1]) / 4));
        col[(size_t)c++].push_back((float)((Jz[i] + Jz[iu]) / 2));
        col[(size_t)c++].push_back((float)((Jr[i] + Jr[ir1]) / 2));
        if (sep) {
          col[(size_t)c++].push_back(ezi);
          col[(size_t)c++].push_back(eri);
        }
      }
      if (te) {
        col[(size_t)c++].push_back((float)Ephi[i]);
        col[(size_t)c++].push_back((float)((Br2[i] + Br2[iu]) / 2));
        col[(size_t)c++].push_back((float)((Bz2[i] + Bz2[ir1]) / 2));
        col[(size_t)c++].push_back((float)Jphi[i]);
      }
    }
  }
  const size_t ncol = 3 + (tm ? 5 + (sep ? 2 : 0) : 0) + (te ? 4 : 0);
  std::vector<const void *> cols;
  for (size_t k = 0; k < ncol; k++)
    cols.push_back(col[k].data());
  const double zdim = std::ceil(nz / (O.z_interval * 1.0)), rdim = std::ceil(nr / (O.r_interval * 1.0));
  std::string err;
  if (!O.out.write_page({m.zmin, m.dz * O.z_interval, zdim, 0.0, m.dr * O.r_interval, rdim, time, (double)step},
                        {}, (int64_t)col[0].size(), cols, err))
    return serr(SPIFFE_ERR_INVALID, "field output: %s", err.c_str());
  return 0;
}

// ------------------------------------------------------------------ integrate

int spiffe_session::ensure_instance()
{
  if (!inst) {
    S_TRY(spiffe_gpu_create(&mesh, flags.data(), precision, particle_capacity, &inst));
    spiffe_field_set f = host_set();
    S_TRY(spiffe_gpu_upload_fields(inst, &f));
    if (precision == SPIFFE_PRECISION_F64)
      S_TRY(spiffe_gpu_set_deposit_order(inst, deposit_order));
    if (precision == SPIFFE_PRECISION_SPLIT32 && poisson_solver >= 0)
      S_TRY(spiffe_gpu_set_poisson_solver(inst, poisson_solver));
  } else {
    S_TRY(spiffe_gpu_set_mesh(inst, &mesh));
  }
  for (SessionCathode &c : cathodes)
    if (!c.on_device) {
      spiffe_cathode_options o = c.o;
      o.n_profile = (int32_t)c.t.size();
      o.profile_t = c.t.empty() ? nullptr : c.t.data();
      o.profile_A = c.A.empty() ? nullptr : c.A.data();
      S_TRY(spiffe_gpu_add_cathode(inst, &o));
      c.on_device = true;
    }
  for (SessionSampling &d : samplings)
    if (d.index < 0)
      S_TRY(spiffe_gpu_add_field_sampling(inst, &d.o, &d.index));
  for (SessionEmitter &e : emitters)
    if (!e.on_device) {
      spiffe_emitter_options o = e.o;
      o.n_points = (int64_t)e.iz.size();
      o.iz = e.iz.data();
      o.ir = e.ir.data();
      o.direction = e.dir.data();
      o.n_profile = (int32_t)e.t.size();
      o.profile_t = e.t.empty() ? nullptr : e.t.data();
      o.profile_A = e.A.empty() ? nullptr : e.A.data();
      S_TRY(spiffe_gpu_add_emitter(inst, &o));
      e.on_device = true;
    }
  if (!secondaries.empty() && !material.empty())
    S_TRY(spiffe_gpu_set_materials(inst, material.data()));
  for (SessionSecondary &d : secondaries)
    if (!d.on_device) {
      spiffe_secondary_options o = d.o;
      o.n_data = (int64_t)d.E.size();
      o.energy = d.E.data();
      o.yield = d.Y.data();
      S_TRY(spiffe_gpu_add_secondary_emission(inst, &o));
      d.on_device = true;
    }
  for (SessionAntenna &an : antennas)
    if (!an.on_device) {
      S_TRY(spiffe_gpu_add_antenna(inst, an.direction, an.istart, an.iend, an.iposition, an.current, an.frequency,
                                   an.phase, an.t.data(), an.W.data(), (int64_t)an.t.size()));
      an.on_device = true;
    }
  for (SessionOnAxis &d : onaxis)
    if (!d.on_device) {
      S_TRY(spiffe_gpu_add_on_axis_field(inst, d.z.data(), d.Ez.data(), (int64_t)d.z.size(), d.z_offset, d.Ez_peak,
                                         d.frequency, d.phase, (int32_t)d.order));
      d.on_device = true;
    }
  for (SessionScreen &sc : screens)
    if (!sc.on_device) {
      S_TRY(spiffe_gpu_add_screen(inst, sc.z, sc.direction, screen_capacity));
      sc.on_device = true;
    }
  S_TRY(spiffe_gpu_set_test_beam(inst, test_beam ? &tb : nullptr));
  if (translate_on && !translate_set) {
    S_TRY(spiffe_gpu_set_translation(inst, 1, z_trigger));
    translate_set = true;
  }
  return 0;
}

// one SDDS page per screen with the records of the steps since the last flush
int spiffe_session::flush_screens(long long step, double time)
{
  bool any = false;
  for (size_t is = 0; is < screens.size(); is++) {
    int64_t nb = 0;
    S_TRY(spiffe_gpu_screen_count(inst, (int32_t)is, &nb));
    if (!nb)
      continue;
    any = true;
    const size_t n = (size_t)nb;
    std::vector<std::vector<double>> q(12, std::vector<double>(n));
    std::vector<int16_t> gen(n);
    std::vector<int32_t> id(n);
    spiffe_screen_set h{};
    h.capacity = nb;
    for (int c = 0; c < SPIFFE_SCREEN_QUANS; c++)
      h.col[c] = q[(size_t)c].data();
    h.rmin = q[8].data();
    h.rmax = q[9].data();
    h.zmin = q[10].data();
    h.zmax = q[11].data();
    h.generation = gen.data();
    h.particleID = id.data();
    S_TRY(spiffe_gpu_download_screen(inst, (int32_t)is, &h));
    std::vector<const void *> cols;
    for (int c = 0; c < 8; c++)
      cols.push_back(q[(size_t)c].data());
    cols.push_back(gen.data());
    cols.push_back(id.data());
    for (int c = 8; c < 12; c++)
      cols.push_back(q[(size_t)c].data());
    std::string err;
    if (!screens[is].out.write_page({time, (double)step}, {"", ""}, nb, cols, err))
      return serr(SPIFFE_ERR_INVALID, "screen %s: %s", screens[is].filename.c_str(), err.c_str());
  }
  if (any)
    S_TRY(spiffe_gpu_clear_screens(inst));
  return 0;
}

// The lost particles since the last flush, written as advance_particles
// writes them (:450-487, :529-535): each step's rows in particle order, in
// pages of at most 1000 rows.
int spiffe_session::flush_lost()
{
  if (!lost_on)
    return 0;
  const size_t cap = (size_t)particle_capacity;
  std::vector<double> t(cap), rl(cap), zl(cap), pz(cap), pr(cap), z0(cap), r0(cap), q(cap);
  std::vector<int16_t> gen(cap);
  std::vector<int32_t> id(cap);
  std::vector<int64_t> step(cap);
  spiffe_lost_set h{0, (int64_t)cap, t.data(), rl.data(), zl.data(), pz.data(), pr.data(), z0.data(), r0.data(),
                    q.data(), gen.data(), id.data(), step.data()};
  S_TRY(spiffe_gpu_download_lost(inst, &h));
  const size_t n = (size_t)h.nb;
  std::vector<float> f[7];
  for (size_t a = 0; a < n;) {
    size_t b = a;
    while (b < n && step[b] == step[a] && b - a < 1000)
      b++;
    const size_t rows = b - a;
    const double *src[7] = {rl.data(), zl.data(), pz.data(), pr.data(), z0.data(), r0.data(), q.data()};
    for (int c = 0; c < 7; c++) {
      f[c].resize(rows);
      for (size_t i = 0; i < rows; i++)
        f[c][i] = (float)src[c][a + i];
    }
    std::vector<const void *> cols = {t.data() + a};
    for (int c = 0; c < 7; c++)
      cols.push_back(f[c].data());
    cols.push_back(gen.data() + a);
    cols.push_back(id.data() + a);
    std::string err;
    if (!lost_out.write_page({}, {}, (int64_t)rows, cols, err))
      return serr(SPIFFE_ERR_INVALID, "lost_particles: %s", err.c_str());
    a = b;
  }
  return 0;
}

// The status file's columns (setUpStatusOutputFile, status_pr.c:454-499):
// the double columns, then Particles, NewParticles, SecondaryParticles
// (long) between ErAbsMax and zMax
static const char *const kStatusD[] = {"t", "JCathode", "KineticEnergy", "FieldEnergy", "TotalEnergy", "Charge",
                                       "EzAbsMax", "ErAbsMax", "zMax", "zMin", "zAve", "zRMS", "zStDev", "rMax",
                                       "rMin", "rAve", "rRMS", "rStDev", "pzMax", "pzMin", "pzAve", "pzRMS",
                                       "pzStDev", "prMax", "prMin", "prAve", "prRMS", "prStDev", "EzOOEMin",
                                       "EzOOEMax"};
static const char *const kStatusDU[] = {"s", "A/m$a2$n", "J", "J", "J", "C", "V/m", "V/m", "m", "m", "m", "m", "m",
                                        "m", "m", "m", "m", "m", "", "", "", "", "", "", "", "", "", "", "V/m", "V/m"};
static const char *const kStatusL[] = {"Particles", "NewParticles", "SecondaryParticles"};

int spiffe_session::status(long long step, double time)
{
  int64_t np = 0, act = 0;
  S_TRY(spiffe_gpu_counts(inst, &np, &act));
  say("step %lld  t=%e s  particles %lld (%lld active)\n", step, time, (long long)np, (long long)act);
  if (!status_on)
    return 0;
  // one row of do_status_printouts (status_pr.c:316-345)
  spiffe_status_row r;
  S_TRY(spiffe_gpu_status_report(inst, &r));
  r.t = time; // the step about to run (integrate.c:138)
  const double d[] = {r.t, r.JCathode, r.KineticEnergy, r.FieldEnergy, r.TotalEnergy, r.Charge, r.EzAbsMax,
                      r.ErAbsMax, r.zMax, r.zMin, r.zAve, r.zRMS, r.zStDev, r.rMax, r.rMin, r.rAve, r.rRMS,
                      r.rStDev, r.pzMax, r.pzMin, r.pzAve, r.pzRMS, r.pzStDev, r.prMax, r.prMin, r.prAve,
                      r.prRMS, r.prStDev, r.EzOOEMin, r.EzOOEMax};
  static_assert(sizeof(d) / sizeof(d[0]) == sizeof(kStatusD) / sizeof(kStatusD[0]), "status columns");
  for (size_t k = 0; k < status_cols.size(); k++)
    status_cols[k].push_back(d[k]);
  status_counts[0].push_back((int32_t)r.Particles);
  status_counts[1].push_back((int32_t)(r.Particles - status_old_np));
  status_counts[2].push_back((int32_t)r.SecondaryParticles);
  status_old_np = r.Particles;
  return write_status();
}

int spiffe_session::write_status()
{
  using namespace spiffe_sdds;
  std::vector<Def> cols;
  std::vector<const void *> ptr;
  for (size_t k = 0; k < status_cols.size(); k++) {
    cols.push_back(Def{kStatusD[k], kStatusDU[k], "", T_DOUBLE});
    ptr.push_back(status_cols[k].data());
    if (k == 7) // after ErAbsMax
      for (int c = 0; c < 3; c++) {
        cols.push_back(Def{kStatusL[c], "", "", T_LONG});
        ptr.push_back(status_counts[(size_t)c].data());
      }
  }
  Writer w;
  std::string err;
  if (!w.open(status_path, "", "", {}, cols, err) ||
      !w.write_page({}, {}, (int64_t)status_counts[0].size(), ptr, err))
    return serr(SPIFFE_ERR_INVALID, "status_output: %s", err.c_str());
  return 0;
}

// perform_integration, integrate.c:24-208
int spiffe_session::cmd_integrate(Args &g)
{
  double dt = 0, start_time = 0, finish_time = 0, smoothing = 0, j_filter = 0, z_forces_start = -1;
  long long status_interval = -1, space_charge = 0, check_divergence = 0, sg = 0, terminate = 0;
  std::string out;
  g.num("dt_integration", dt);
  g.num("start_time", start_time);
  g.num("finish_time", finish_time);
  g.integer("status_interval", status_interval);
  g.integer("space_charge", space_charge);
  g.integer("check_divergence", check_divergence); // changes only the status report
  g.num("smoothing_parameter", smoothing);
  g.num("j_filter_multiplier", j_filter);
  g.integer("sg_smoothing_halfwidth", sg);
  g.integer("terminate_on_total_loss", terminate);
  g.num("z_forces_start", z_forces_start);
  std::string status_output;
  const bool have_status = g.str("status_output", status_output);
  std::string lost_particles;
  const bool have_lost = g.str("lost_particles", lost_particles);
  g.num("imposed_efield_ramp_time", ramp_time);
  g.num("imposed_efield_flat_top_time", flat_top_time);
  g.integer("auto_max_dt", auto_max_dt);
  S_TRY(g.finish());
  if (!have_geometry)
    return serr(SPIFFE_ERR_INVALID, "integrate before define_geometry");
  if (dt <= 0)
    return serr(SPIFFE_ERR_INVALID, "dt_integration <= 0");
  if (finish_time < start_time)
    return serr(SPIFFE_ERR_INVALID, "finish_time < start_time");
  if (smoothing < 0 || smoothing > 1)
    return serr(SPIFFE_ERR_INVALID, "smoothing_parameter must be >= 0 and < 1");
  if (j_filter < 0 || j_filter >= 1)
    return serr(SPIFFE_ERR_INVALID, "J_filter_multiplier must be >=0 and < 1");
  if (smoothing || j_filter || sg)
    return serr(SPIFFE_ERR_UNSUPPORTED, "integrate: current smoothing and filtering are not supported");
  // setUpLostParticleFile, advance_particles.c:577-603 (integrate.c:81-82)
  lost_on = have_lost && !lost_particles.empty();
  if (lost_on) {
    using namespace spiffe_sdds;
    lost_path = compose(lost_particles, rootname);
    const std::vector<Def> cols = {Def{"t", "s", "", T_DOUBLE},    Def{"rLost", "m", "", T_FLOAT},
                                   Def{"zLost", "m", "", T_FLOAT}, Def{"pz", "", "", T_FLOAT},
                                   Def{"pr", "", "", T_FLOAT},     Def{"z0", "m", "", T_FLOAT},
                                   Def{"r0", "m", "", T_FLOAT},    Def{"q", "C", "", T_FLOAT},
                                   Def{"generation", "", "", T_SHORT}, Def{"particleID", "", "", T_LONG}};
    std::string err;
    if (!lost_out.open(lost_path, "", "", {}, cols, err))
      return serr(SPIFFE_ERR_INVALID, "lost_particles: %s", err.c_str());
  }
  // setUpStatusOutputFile, status_pr.c:454-499 (integrate.c:79-80)
  status_on = have_status && !status_output.empty();
  if (status_on) {
    status_path = compose(status_output, rootname);
    status_cols.assign(sizeof(kStatusD) / sizeof(kStatusD[0]), {});
    status_counts.assign(3, {});
    status_old_np = 0;
    S_TRY(write_status());
  }
  if (inst)
    S_TRY(spiffe_gpu_get_mesh(inst, &mesh));
  spiffe_mesh &m = mesh;
  const bool is_reload = m.dt != 0;
  if (space_charge)
    m.modes |= SPIFFE_FL_SPACE_CHARGE;
  m.imposed_ramp_time = ramp_time;
  m.imposed_flat_top_time = flat_top_time;
  m.dt = dt;
  if (!is_reload)
    m.start_time = start_time;
  else
    start_time = m.start_time;
  long long n_steps = (long long)((finish_time - start_time) / dt);
  const double dtC = std::fmin(m.dz, m.dr) / SPIFFE_C_MKS / std::sqrt(2.0);
  if (dtC < m.dt) {
    if (!auto_max_dt)
      return serr(SPIFFE_ERR_INVALID, "the time step must be less than %es for stable integration.", dtC);
    warn("dt_integration (%e) exceeds max stable dt (%e); using max dt", dt, dtC);
    m.dt = dtC;
    n_steps = (long long)((finish_time - start_time) / m.dt);
  }
  S_TRY(ensure_instance());
  const int sc = (m.modes & SPIFFE_FL_SPACE_CHARGE) ? 1 : 0;
  spiffe_push_options push{};
  push.z_forces_start = z_forces_start;
  push.tb_electrons_per_macroparticle = test_beam ? tb.electrons_per_macroparticle : 0;
  push.tb_z_force = tb_z_force;
  push.tb_r_force = tb_r_force;
  push.tb_z_start_deceleration = tb_z_decel;
  push.tb_r_start_deceleration = tb_r_decel;
  const bool f64 = precision == SPIFFE_PRECISION_F64;
  push.compaction = compaction >= 0 ? compaction : (f64 ? SPIFFE_COMPACT_REFERENCE : SPIFFE_COMPACT_ANY);
  push.screen_momentum = screen_momentum >= 0 ? screen_momentum : (f64 ? SPIFFE_SCREEN_REFERENCE : SPIFFE_SCREEN_PARTICLE);
  S_TRY(spiffe_gpu_configure_run(inst, sc, &push, pc_defined ? &pc : nullptr));
  S_TRY(spiffe_gpu_set_lost_log(inst, lost_on ? particle_capacity : 0));
  S_TRY(spiffe_gpu_run_begin(inst, nullptr));
  say("integration will consist of up to %lld steps spaced by %e\n", n_steps, m.dt);

  S_TRY(spiffe_gpu_get_mesh(inst, &m));
  long long k = m.time_step;
  const spiffe_poisson_options no_pc{};
  const double t0 = m.start_time, step_dt = m.dt;
  bool beam_seen = false;
  auto next_save = [&](long long from) -> long long {
    if (!saving.defined || saving.save_index == -1)
      return from;
    return next_due(from, saving.start_step, saving.step_interval);
  };
  while (k < n_steps) {
    const double t = k * step_dt + t0;
    if (terminate) {
      int64_t np = 0;
      S_TRY(spiffe_gpu_counts(inst, &np, nullptr));
      if (beam_seen && !np) {
        say("simulation terminating due to total loss of particles.\n");
        break;
      }
      if (np && !beam_seen)
        beam_seen = true;
    }
    // the step's imposed-field ramp comes before the diagnostics
    // (integrate.c:136-137); run_steps then finds the factor unchanged
    if (m.imposed_ramp_time > 0) {
      bool need = status_on && status_interval > 0 && k % status_interval == 0;
      if (field_output.defined) {
        const bool first = field_output.index == -1; // the schedule is fixed at the first output call
        const long long fs = first ? (long long)((field_output.start_time - m.start_time) / m.dt + 0.5)
                                   : field_output.start_step;
        const long long fi = first ? (long long)(field_output.time_interval / m.dt + 0.5) : field_output.step_interval;
        need = need || due(k, fs, fi);
      }
      if (need)
        S_TRY(spiffe_gpu_compute_imposed_efield(inst, pc_defined ? &pc : &no_pc, 0));
    }
    S_TRY(save_fields(k, t, false));
    S_TRY(output_fields(k, t));
    S_TRY(take_snapshot(k, t));
    if (status_interval > 0 && k % status_interval == 0)
      S_TRY(status(k, t));
    long long next = n_steps;
    if (terminate)
      next = k + 1;
    if (flush_steps > 0 && k + flush_steps < next)
      next = k + flush_steps;
    if (saving.defined) {
      const long long s = next_save(k + 1);
      if (s < next)
        next = s;
    }
    if (snapshots.defined) {
      const long long s = next_due(k + 1, snapshots.start_step, snapshots.step_interval);
      if (s < next)
        next = s;
    }
    if (field_output.defined) {
      const long long s = next_due(k + 1, field_output.start_step, field_output.step_interval);
      if (s < next)
        next = s;
    }
    if (status_interval > 0) {
      const long long s = (k / status_interval + 1) * status_interval;
      if (s < next)
        next = s;
    }
    S_TRY(spiffe_gpu_run_steps(inst, next - k));
    steps += next - k;
    S_TRY(flush_screens(next - 1, (next - 1) * step_dt + t0));
    S_TRY(flush_lost());
    S_TRY(flush_secondary_logs());
    S_TRY(flush_samples());
    k = next;
  }
  if (lost_on) { // SDDS_Terminate, integrate.c:203
    lost_out.close();
    lost_on = false;
    S_TRY(spiffe_gpu_set_lost_log(inst, 0));
  }
  // integrate.c:195-206
  S_TRY(spiffe_gpu_get_mesh(inst, &m));
  m.time = m.time_step * m.dt + m.start_time;
  S_TRY(spiffe_gpu_set_mesh(inst, &m));
  S_TRY(spiffe_gpu_sample_fields(inst));
  S_TRY(flush_samples());
  S_TRY(save_fields(m.time_step, m.time, true));
  S_TRY(take_snapshot(m.time_step, m.time));
  if (status_interval > 0 && m.time_step % status_interval == 0)
    S_TRY(status(m.time_step, m.time));
  return 0;
}

// ------------------------------------------------------------------- dispatch

// the command loop of spiffe.c:213-308
int spiffe_session::execute(const std::string &text)
{
  size_t pos = 0;
  std::string err;
  Args g;
  while (spiffe_nl::next_block(text, pos, g.group, g.e, err)) {
    g.used.assign(g.e.size(), 0);
    g.bad.clear();
    const std::string &c = g.group;
    say("&%s\n", c.c_str());
    int rc;
    if (c == "define_geometry")
      rc = cmd_geometry(g);
    else if (c == "set_constant_fields" || c == "constant_fields")
      rc = cmd_constant_fields(g);
    else if (c == "define_solenoid")
      rc = cmd_solenoid(g);
    else if (c == "define_cathode")
      rc = cmd_cathode(g);
    else if (c == "define_antenna")
      rc = cmd_antenna(g);
    else if (c == "add_on_axis_fields")
      rc = cmd_on_axis_fields(g);
    else if (c == "define_screen")
      rc = cmd_screen(g);
    else if (c == "define_test_beam")
      rc = cmd_test_beam(g);
    else if (c == "poisson_correction")
      rc = cmd_poisson(g);
    else if (c == "load_fields")
      rc = cmd_load_fields(g);
    else if (c == "define_field_saving")
      rc = cmd_field_saving(g);
    else if (c == "integrate")
      rc = cmd_integrate(g);
    else if (c == "trace") {
      warn("trace feature is obsolete and no longer available");
      rc = 0;
    } else if (c == "stop") {
      return SPIFFE_SESSION_STOPPED;
    } else if (c == "space_charge") {
      rc = serr(SPIFFE_ERR_INVALID, "the space_charge namelist is no longer used--use space_charge=1 in the integrate namelist");
    } else if (c == "define_snapshots") {
      rc = cmd_snapshots(g);
    } else if (c == "define_field_output") {
      rc = cmd_field_output(g);
    } else if (c == "define_field_sampling") {
      rc = cmd_field_sampling(g);
    } else if (c == "translate") {
      rc = cmd_translate(g);
    } else if (c == "define_secondary_emission") {
      rc = cmd_secondary_emission(g);
    } else if (c == "define_emitter") {
      rc = cmd_emitter(g);
    } else if (c == "define_resistor" || c == "load_particles") {
      rc = serr(SPIFFE_ERR_UNSUPPORTED, "%s is not supported", c.c_str());
    } else {
      rc = serr(SPIFFE_ERR_INVALID, "unknown namelist %s given", c.c_str());
    }
    if (rc < 0)
      return rc;
  }
  if (!err.empty())
    return serr(SPIFFE_ERR_INVALID, "%s", err.c_str());
  return 0;
}

// --------------------------------------------------------------- solenoid

namespace {

// Complete elliptic integrals K(k) and E(k) by the arithmetic-geometric mean
// (Abramowitz & Stegun 17.6.3-17.6.4): a, b -> (a+b)/2, sqrt(ab) from 1,
// sqrt(1-k^2); K = pi/(2 a_inf); E = K (1 - sum 2^(n-1) c_n^2), c_0 = k.
void agm_elliptic(double k, double *K, double *E)
{
  double a = 1, b = std::sqrt(1 - k * k), c = k, sum = 0.5 * k * k, w = 0.5;
  for (int n = 0; n < 60 && std::fabs(c) > 1e-17; n++) {
    const double an = (a + b) / 2;
    c = (a - b) / 2;
    b = std::sqrt(a * b);
    a = an;
    w *= 2;
    sum += w * c * c;
  }
  *K = SPIFFE_PI / (2 * a);
  *E = *K * (1 - sum);
}

// Field of a 1 A circular loop of radius R at (rho, z) relative to its
// centre (Landau & Lifshitz, Electrodynamics of Continuous Media, section 30),
// mu0/(2 pi) = 2e-7; the reference evaluates it as Bsolenoid.c:56-86 does.
void ring_field(double rho, double z, double R, double *Brho, double *Bz)
{
  const double z2 = z * z;
  const double s1 = R * R + rho * rho + z2;
  const double s2 = R * R - rho * rho - z2;
  const double ap = R + rho, am = R - rho;
  const double s3 = ap * ap + z2;
  const double s4 = am * am + z2;
  double K, E;
  agm_elliptic(std::sqrt(4 * R * rho / s3), &K, &E);
  const double F = 2e-7 / std::sqrt(s3);
  *Brho = rho ? F * z / rho * (-K + E * s1 / s4) : 0;
  *Bz = F * (K + E * s2 / s4);
}

// `coils` rings evenly from z_start to z_end, B_solenoid of Bsolenoid.c:17-49
void coil_field(double rho, double z, double R, double z_start, double z_end, long long coils, int symmetry,
                double *Brho, double *Bz)
{
  *Brho = *Bz = 0;
  const double dzc = coils > 1 ? (z_end - z_start) / (coils - 1) : 0;
  for (long long i = 0; i < coils; i++) {
    const double zc = z_start + i * dzc;
    double br, bz;
    ring_field(rho, z - zc, R, &br, &bz);
    *Brho += br;
    *Bz += bz;
    if (symmetry && zc) {
      ring_field(rho, z + zc, R, &br, &bz);
      if (symmetry == 1) {
        *Brho += br;
        *Bz += bz;
      } else {
        *Brho -= br;
        *Bz -= bz;
      }
    }
  }
}

} // namespace

extern "C" int spiffe_solenoid_add(const spiffe_mesh *mesh, const spiffe_solenoid_options *o, double *Bz, double *Br,
                                   double *current_used)
{
  if (!mesh || !o || !Bz || !Br)
    return serr(SPIFFE_ERR_INVALID, "null argument");
  if (o->radius <= 0)
    return serr(SPIFFE_ERR_INVALID, "radius <= 0 is not valid");
  if (o->evaluation_radius_limit < 0)
    return serr(SPIFFE_ERR_INVALID, "evaluation_radius_limit < 0  is not valid");
  if (o->z_start > o->z_end)
    return serr(SPIFFE_ERR_INVALID, "z_start > z_end is not valid");
  if (o->turns <= 0)
    return serr(SPIFFE_ERR_INVALID, "turns <= 0 is not valid");
  if (o->symmetry && o->symmetry != -1 && o->symmetry != 1)
    return serr(SPIFFE_ERR_INVALID, "symmetry must be 0, 1, or -1");
  const long long nz = mesh->nz, nr = mesh->nr, P = nr + 1;
  long long nr_limit = nr;
  if (o->evaluation_radius_limit && (nr_limit = (long long)(o->evaluation_radius_limit / mesh->dr + 0.5)) > nr)
    nr_limit = nr;
  double current = o->current;
  if (o->bucking) {
    // solenoid.c:66-79: the current that cancels the on-axis Bz at z_buck
    const long long iz = (long long)((o->z_buck - mesh->zmin) / mesh->dz);
    if (iz < 0 || iz > nz)
      return serr(SPIFFE_ERR_INVALID, "z_buck is outside of simulation region");
    double br1, bz1;
    coil_field(0.0, o->z_buck, o->radius, o->z_start, o->z_end, o->turns, o->symmetry, &br1, &bz1);
    current = bz1 != 0 ? -Bz[iz * P] / bz1 : 0;
  }
  double z = mesh->zmin;
  for (long long iz = 0; iz <= nz; iz++) {
    double r = 0;
    for (long long ir = 0; ir <= nr_limit; ir++) {
      double br1, bz1;
      coil_field(r, z, o->radius, o->z_start, o->z_end, o->turns, o->symmetry, &br1, &bz1);
      Br[iz * P + ir] += br1 * current;
      Bz[iz * P + ir] += bz1 * current;
      r += mesh->dr;
    }
    z += mesh->dz;
  }
  if (o->Bz_peak) {
    double bmax = -DBL_MAX;
    long long izm = -1;
    for (long long iz = 0; iz <= nz; iz++)
      if (Bz[iz * P] > bmax) {
        izm = iz;
        bmax = Bz[iz * P];
      }
    if (izm == -1)
      return serr(SPIFFE_ERR_INVALID, "problem scaling solenoid fields to Bz_peak---didn't find maximum!");
    if (bmax == 0)
      return serr(SPIFFE_ERR_INVALID, "problem scaling solenoid fields to Bz_peak---maximum field is zero");
    for (long long iz = 0; iz <= nz; iz++)
      for (long long ir = 0; ir <= nr_limit; ir++) {
        Bz[iz * P + ir] *= o->Bz_peak / bmax;
        Br[iz * P + ir] *= o->Bz_peak / bmax;
      }
  }
  if (current_used)
    *current_used = current;
  return 0;
}

// ------------------------------------------------------------------- C ABI

extern "C" int spiffe_session_create(int32_t precision, const char *rootname, spiffe_session **out)
{
  if (!out)
    return serr(SPIFFE_ERR_INVALID, "null argument");
  if (precision != SPIFFE_PRECISION_F64 && precision != SPIFFE_PRECISION_SPLIT32)
    return serr(SPIFFE_ERR_INVALID, "unknown precision %d", precision);
  spiffe_session *s = new spiffe_session;
  s->precision = precision;
  if (rootname && *rootname)
    s->rootname = rootname;
  *out = s;
  return 0;
}

extern "C" int spiffe_session_destroy(spiffe_session *s)
{
  if (!s)
    return 0;
  int rc = 0;
  if (s->inst)
    rc = spiffe_gpu_destroy(s->inst);
  delete s;
  return rc;
}

extern "C" int spiffe_session_execute(spiffe_session *s, const char *text)
{
  if (!s || !text)
    return serr(SPIFFE_ERR_INVALID, "null argument");
  return s->execute(text);
}

extern "C" int spiffe_session_run_file(spiffe_session *s, const char *path)
{
  if (!s || !path)
    return serr(SPIFFE_ERR_INVALID, "null argument");
  std::string text, err;
  if (!read_text(path, text, err))
    return serr(SPIFFE_ERR_INVALID, "%s", err.c_str());
  s->run_name = path;
  return s->execute(text);
}

extern "C" int spiffe_session_set(spiffe_session *s, const char *name, double v)
{
  if (!s || !name)
    return serr(SPIFFE_ERR_INVALID, "null argument");
  const std::string n = name;
  if (n == "verbose")
    s->verbose = (int)v;
  else if (n == "deposit_order")
    s->deposit_order = (int)v;
  else if (n == "particle_capacity" && v > 0)
    s->particle_capacity = (long long)v;
  else if (n == "screen_capacity" && v > 0)
    s->screen_capacity = (long long)v;
  else if (n == "flush_steps" && v > 0)
    s->flush_steps = (long long)v;
  else if (n == "compaction" && v >= 0 && v <= 2)
    s->compaction = (int)v;
  else if (n == "screen_momentum" && v >= 0 && v <= 1)
    s->screen_momentum = (int)v;
  else if (n == "poisson_solver" && (v == SPIFFE_POISSON_SOR || v == SPIFFE_POISSON_MULTIGRID))
    s->poisson_solver = (int)v;
  else
    return serr(SPIFFE_ERR_INVALID, "unknown session setting %s or bad value", name);
  if (s->inst && n == "deposit_order" && s->precision == SPIFFE_PRECISION_F64)
    return spiffe_gpu_set_deposit_order(s->inst, s->deposit_order);
  return 0;
}

extern "C" int spiffe_session_mesh(spiffe_session *s, spiffe_mesh *mesh)
{
  if (!s || !mesh)
    return serr(SPIFFE_ERR_INVALID, "null argument");
  if (!s->have_geometry)
    return serr(SPIFFE_ERR_INVALID, "no geometry defined");
  if (s->inst)
    S_TRY(spiffe_gpu_get_mesh(s->inst, &s->mesh));
  *mesh = s->mesh;
  return 0;
}

extern "C" int spiffe_session_fields(spiffe_session *s, spiffe_field_set *h)
{
  if (!s || !h)
    return serr(SPIFFE_ERR_INVALID, "null argument");
  if (!s->have_geometry)
    return serr(SPIFFE_ERR_INVALID, "no geometry defined");
  S_TRY(s->pull());
  const size_t n = s->nodes();
  for (const char *name : kFieldNames) {
    double *dst = *slot(*h, name);
    if (dst && s->has(name))
      std::memcpy(dst, s->a[name].data(), n * sizeof(double));
  }
  if (h->flags)
    std::memcpy(h->flags, s->flags.data(), n * sizeof(int16_t));
  return 0;
}

extern "C" int spiffe_session_instance(spiffe_session *s, spiffe_gpu_instance **inst)
{
  if (!s || !inst)
    return serr(SPIFFE_ERR_INVALID, "null argument");
  *inst = s->inst;
  return 0;
}

extern "C" int64_t spiffe_session_steps(spiffe_session *s) { return s ? s->steps : 0; }
