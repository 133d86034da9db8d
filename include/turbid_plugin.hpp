/* C++ host layer over the C ABI of libturbid_gpu.so: the plugin classes of the
 * reference's flat-channel solver (yueliangyi/TURBID), same names, same method
 * meaning, same "Class::Method > message" std::runtime_error convention.
 *
 *   IniFile              src/file_ini.cc:43-112 (Load), :241-292 (values)
 *   RK3TimeStepper       src/stepper_time_rk3.cc:28-31, src/stepper_time.cc:72-113
 *   FlatCarrierPhase     src/phase_carrier_flat.cc:178-994 (Predict/Correct on the GPU)
 *   FlatScalarPhase      src/phase_scalar_flat.cc:176-667
 *   FlatCarrierVariable  src/variable_carrier_flat.cc:143-377 (Save/Load, IO level one)
 *   FlatChannelSolver    src/solver_channel_flat.cc:31-120 (Configure), :199-293
 *                        (Execute), :372-414 (PrintLogBody)
 *   FlatChannelPostprocessor  src/postprocessor_channel_flat.cc:153-236 (swirling
 *                        strength of the saved states, phase_00_vortex.dat)
 *
 * One GPU context (tg_ctx) holds the whole case; the phase objects are views
 * on it that call the per-stage entry points, so the Execute loop below is the
 * reference's loop with the phase bodies running on the GPU.  Header-only;
 * link with -lturbid_gpu.
 */
#pragma once

#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "turbid_gpu.h"

namespace turbid {

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
inline void Check(const std::string& where, tg_status st) {
  if (st != TG_OK) throw std::runtime_error(where + " > " + tg_last_error());
}

// ---------------------------------------------------------------------------
// Arithmetic expressions of .ini values ("2*pi/12000", "10E+6", "8*pi"):
// + - * / % ^, unary signs, parentheses, pi and e, and the functions sin cos
// tan exp log sqrt abs atan asin acos sinh cosh tanh pow.  A recursive-descent
// evaluator of our own (the reference uses exprtk).
// ---------------------------------------------------------------------------
class Expression {
 public:
  static double Evaluate(const std::string& text) {
    Expression e(text);
    const double v = e.Sum();
    e.Skip();
    if (e.p_ != e.s_.size()) e.Fail();
    return v;
  }

 private:
  explicit Expression(const std::string& s) : s_(s) {}
  [[noreturn]] void Fail() const {
    throw std::runtime_error("IniFile::GetValueDouble > Can not Evaluate Expression: " + s_);
  }
  void Skip() {
    while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_;
  }
  bool Eat(char c) {
    Skip();
    if (p_ < s_.size() && s_[p_] == c) {
      ++p_;
      return true;
    }
    return false;
  }
  double Sum() {
    double v = Product();
    for (;;) {
      if (Eat('+')) v += Product();
      else if (Eat('-')) v -= Product();
      else return v;
    }
  }
  double Product() {
    double v = Unary();
    for (;;) {
      if (Eat('*')) v *= Unary();
      else if (Eat('/')) v /= Unary();
      else if (Eat('%')) v = std::fmod(v, Unary());
      else return v;
    }
  }
  double Unary() {
    if (Eat('-')) return -Unary();
    if (Eat('+')) return Unary();
    return Power();
  }
  double Power() {  // right associative, binds tighter than unary minus on its left
    const double b = Atom();
    if (Eat('^')) return std::pow(b, Unary());
    return b;
  }
  double Atom() {
    Skip();
    if (p_ >= s_.size()) Fail();
    if (Eat('(')) {
      const double v = Sum();
      if (!Eat(')')) Fail();
      return v;
    }
    const char c = s_[p_];
    if (std::isdigit((unsigned char)c) || c == '.') {
      const char* begin = s_.c_str() + p_;
      char* end = nullptr;
      const double v = std::strtod(begin, &end);
      if (end == begin) Fail();
      p_ += (size_t)(end - begin);
      return v;
    }
    if (std::isalpha((unsigned char)c)) {
      size_t q = p_;
      while (q < s_.size() && (std::isalnum((unsigned char)s_[q]) || s_[q] == '_')) ++q;
      std::string name = s_.substr(p_, q - p_);
      std::transform(name.begin(), name.end(), name.begin(), ::tolower);
      p_ = q;
      if (name == "pi") return 3.14159265358979323846;
      if (name == "e") return 2.71828182845904523536;
      if (!Eat('(')) Fail();
      std::vector<double> a{Sum()};
      while (Eat(',')) a.push_back(Sum());
      if (!Eat(')')) Fail();
      if (name == "pow" && a.size() == 2) return std::pow(a[0], a[1]);
      if (a.size() != 1) Fail();
      const double x = a[0];
      if (name == "sin") return std::sin(x);
      if (name == "cos") return std::cos(x);
      if (name == "tan") return std::tan(x);
      if (name == "exp") return std::exp(x);
      if (name == "log") return std::log(x);
      if (name == "sqrt") return std::sqrt(x);
      if (name == "abs") return std::fabs(x);
      if (name == "atan") return std::atan(x);
      if (name == "asin") return std::asin(x);
      if (name == "acos") return std::acos(x);
      if (name == "sinh") return std::sinh(x);
      if (name == "cosh") return std::cosh(x);
      if (name == "tanh") return std::tanh(x);
    }
    Fail();
  }
  std::string s_;
  size_t p_ = 0;
};

// ---------------------------------------------------------------------------
// IniFile: "[Section]" and "key = value" lines, ';' and '#' comments, exact
// case (the reference's solver loads it with SetSensitive(0)).
// ---------------------------------------------------------------------------
class IniFile {
 public:
  void Load(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("IniFile::Load > Can not Open File: " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    Parse(ss.str());
  }
  void Parse(const std::string& text) {
    std::istringstream in(text);
    std::string line, sec;
    while (std::getline(in, line)) {
      const size_t p = line.find_first_of(";#[=");
      if (p == std::string::npos) continue;
      if (line[p] == '[') {
        const size_t r = line.rfind(']');
        if (r != std::string::npos && r > p) {
          sec = Trim(line.substr(p + 1, r - p - 1));
          sections_[sec];
        }
      } else if (line[p] == '=') {
        std::string val = line.substr(p + 1);
        const size_t c = val.find_first_of(";#");
        if (c != std::string::npos) val = val.substr(0, c);
        sections_[sec][Trim(line.substr(0, p))] = Trim(val);
      }
    }
  }
  const std::string& GetValueString(const std::string& sec, const std::string& key) const {
    auto s = sections_.find(sec);
    if (s == sections_.end()) throw std::runtime_error("IniFile::GetValueString > Can not Find Section: " + sec);
    auto k = s->second.find(key);
    if (k == s->second.end())
      throw std::runtime_error("IniFile::GetValueString > Can not Find Key: " + key + " in Section " + sec);
    return k->second;
  }
  int GetValueInt(const std::string& sec, const std::string& key) const {
    return std::stoi(GetValueString(sec, key));
  }
  double GetValueDouble(const std::string& sec, const std::string& key) const {
    return Expression::Evaluate(GetValueString(sec, key));
  }
  std::vector<double> GetVectorDouble(const std::string& sec, const std::string& key) const {
    std::istringstream in(GetValueString(sec, key));
    std::vector<double> v;
    std::string tok;
    while (in >> tok) v.push_back(Expression::Evaluate(tok));
    return v;
  }
  bool HasKey(const std::string& sec, const std::string& key) const {
    auto s = sections_.find(sec);
    return s != sections_.end() && s->second.count(key) != 0;
  }
  std::vector<int> GetVectorInt(const std::string& sec, const std::string& key) const {
    std::istringstream in(GetValueString(sec, key));
    std::vector<int> v;
    std::string tok;
    while (in >> tok) v.push_back(std::stoi(tok));
    return v;
  }

 private:
  static std::string Trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
  }
  std::map<std::string, std::map<std::string, std::string>> sections_;
};

inline std::string Upper(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), ::toupper);
  return s;
}

// ---------------------------------------------------------------------------
// Run control of [Time Stepper] (the fixed-dt branch, output_based_on_step = 1)
// ---------------------------------------------------------------------------
struct RunControl {
  int maxstep = 0, writeinterval = 1, startstep = 0, output_based_on_step = 1;
  double maxcfl = 1.0;
  // adaptive-dt branch (output_based_on_step = 0), src/stepper_time.cc:31-37
  double max_marching_time = 0, output_interval = 0, initial_time_step = 0;
  int start_time_index = -1;
  double cfl_adjust_scale[2] = {0.95, 0.9};
};

// The tg_case fields and run control from a configuration file (the keys of
// src/configure.h:51-118 that the flat-bottom RK3 path reads).
inline tg_case CaseFromIni(const IniFile& ini, RunControl& rc, int precision = TG_PREC_FP64) {
  tg_case c{};
  const std::vector<int> n = ini.GetVectorInt("Domain", "grid_point_number");
  if (n.size() != 3) throw std::runtime_error("Domain::Configuration::Load(IniFile) > grid_point_number needs 3 values");
  c.nx = n[0];
  c.ny = n[1];
  c.nz = n[2];
  const std::vector<double> len = ini.GetVectorDouble("Domain", "dimensionless_length");
  if (len.size() != 3) throw std::runtime_error("Domain::Configuration::Load(IniFile) > dimensionless_length needs 3 values");
  if (std::fabs(len[2] - 2.0) > 10e-12)
    throw std::runtime_error("Domain::Domain > Dimensionless z-length Should be Equal to Two!");
  c.lx = len[0];
  c.ly = len[1];
  c.slope = ini.GetValueDouble("Domain", "top_bottom_slope");
  c.slope_direction = ini.GetValueInt("Domain", "slope_direction");
  c.nphase = ini.GetValueInt("System", "total_phase_number");
  if (Upper(ini.GetValueString("Space Stepper", "applied_stepper_type")) != "CHEBYSHEV")
    throw std::runtime_error("FlatChannelSolver::FlatChannelSolver > Only the Chebyshev Space Stepper is Supported!");
  const std::string mf = Upper(ini.GetValueString("Space Stepper", "mapping_function"));
  if (mf == "NONE") c.mapping = 0;
  else if (mf == "TWOENDTANGENT") c.mapping = 1;
  else if (mf == "TWOENDSIN") c.mapping = 2;
  else if (mf == "ONEENDTANGENT") c.mapping = 3;
  else throw std::runtime_error("SpaceStepper::Configuration::Load(IniFile) > Unsupported Mapping Function!");
  c.mapping_coef = ini.GetVectorDouble("Space Stepper", "mapping_coefficient").at(0);
  if (Upper(ini.GetValueString("Time Stepper", "applied_stepper_type")) != "RUNGEKUTTA3")
    throw std::runtime_error("FlatChannelSolver::FlatChannelSolver > Only the RungeKutta3 Time Stepper is Supported!");
  c.dt = ini.GetValueDouble("Time Stepper", "marching_time_step");
  c.output_based_on_step = ini.GetValueInt("Time Stepper", "output_based_on_step");
  rc.output_based_on_step = c.output_based_on_step;
  rc.maxcfl = ini.GetValueDouble("Time Stepper", "maximum_cfl_number");
  rc.maxstep = ini.GetValueInt("Time Stepper", "maximum_task_step");
  rc.writeinterval = ini.GetValueInt("Time Stepper", "result_write_interval");
  rc.startstep = ini.GetValueInt("Time Stepper", "task_start_step");
  if (rc.output_based_on_step == 0) {
    rc.max_marching_time = ini.GetValueDouble("Time Stepper", "max_marching_time");
    rc.output_interval = ini.GetValueDouble("Time Stepper", "output_interval");
    rc.initial_time_step = ini.GetValueDouble("Time Stepper", "initial_time_step");
    rc.start_time_index = ini.GetValueInt("Time Stepper", "task_start_time_index");
    const std::vector<double> adj = ini.GetVectorDouble("Time Stepper", "cfl_adjust_scale");
    if (adj.size() < 2) throw std::runtime_error("TimeStepper::Configuration::Load(IniFile) > cfl_adjust_scale needs 2 values");
    rc.cfl_adjust_scale[0] = adj[0];
    rc.cfl_adjust_scale[1] = adj[1];
    c.dt = rc.initial_time_step;  // the solves are assembled for the first dt
  }
  const std::string s = "Phase Carrier";
  const std::string ft = Upper(ini.GetValueString(s, "applied_force_type"));
  if (ft == "NONE") c.force_type = 0;
  else if (ft == "CONSTANT") c.force_type = 1;
  else if (ft == "OSCILLATORY") c.force_type = 2;
  else if (ft == "PULSATILE") c.force_type = 3;
  else if (ft == "DAMPING") c.force_type = 4;
  else throw std::runtime_error("FlatCarrierPhase::Configuration::Load(IniFile) > Unsupported Force Type!");
  const std::vector<double> fd = ini.GetVectorDouble(s, "force_direction");
  const std::vector<double> fa = ini.GetVectorDouble(s, "force_amplitude");
  for (size_t i = 0; i < 2 && i < fd.size(); ++i) c.force_direction[i] = (int)fd[i];
  for (size_t i = 0; i < 4 && i < fa.size(); ++i) c.force_amplitude[i] = fa[i];
  c.reynolds = ini.GetValueDouble(s, "reynolds_number");
  c.froude = ini.GetValueDouble(s, "froude_number");
  c.averaged_concentration = ini.GetValueDouble(s, "averaged_concentration");
  c.specific_gravity = ini.GetValueDouble(s, "specific_gravity");
  c.affected_by_scalar = ini.GetValueInt(s, "affected_by_scalar_phase");
  const char* bck[4] = {"vertical_type_u1", "vertical_type_u2", "vertical_type_u3", "vertical_type_p"};
  double* bcs[4] = {c.bc_u, c.bc_v, c.bc_w, c.bc_p};
  for (int i = 0; i < 4; ++i) {
    const std::vector<double> v = ini.GetVectorDouble(s, bck[i]);
    if (v.size() != 5) throw std::runtime_error(std::string("FlatCarrierPhase::Configuration::Load(IniFile) > ") + bck[i] + " needs 5 values");
    for (int k = 0; k < 5; ++k) bcs[i][k] = v[k];
  }
  c.scalar_bc = 0;
  if (c.nphase > 1) {
    const std::string t = "Phase Scalar";
    c.schmidt = ini.GetValueDouble(t, "schmidt_number");
    c.settling = ini.GetValueDouble(t, "settling_velocity");
    c.erosion_rate = ini.GetValueDouble(t, "erosion_rate");
    const std::string bt = Upper(ini.GetValueString(t, "vertical_boundary_type"));
    if (bt == "ZEROFLUX") {
      c.scalar_bc = 0;
    } else if (bt == "EROSIONDEPOSITION") {
      c.scalar_bc = 1;
      c.critical_shear = ini.GetVectorDouble(t, "critical_shear_stress").at(0);
    } else {
      throw std::runtime_error("FlatScalarPhase::Configuration::Load(IniFile) > Unsupported Boundary Type!");
    }
  }
  c.precision = precision;
  return c;
}

// ---------------------------------------------------------------------------
// Restart files: "IOControlLevelOne\n" then Armadillo binary complex cubes
// ("ARMA_CUB_BIN_FC016\n<Nz> <Nyc> <Nxh*dim>\n" + FP64 complex data, z fastest)
// ---------------------------------------------------------------------------
inline void WriteCube(std::ostream& f, const std::vector<std::complex<double>>& v, int nz, int nyc, int nslices) {
  f << "ARMA_CUB_BIN_FC016\n" << nz << " " << nyc << " " << nslices << "\n";
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(v[0])));
}

inline std::vector<std::complex<double>> ReadCube(std::istream& f, int nz, int nyc, int nslices,
                                                  const std::string& where) {
  std::string head;
  std::getline(f, head);
  if (head != "ARMA_CUB_BIN_FC016") throw std::runtime_error(where + " > Not an Armadillo Complex Cube");
  int a = 0, b = 0, c = 0;
  std::string dims;
  std::getline(f, dims);
  std::istringstream(dims) >> a >> b >> c;
  if (a != nz || b != nyc || c != nslices) throw std::runtime_error(where + " > Cube Size Does not Match the Case");
  std::vector<std::complex<double>> v((size_t)nz * nyc * nslices);
  f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(v.size() * sizeof(v[0])));
  if (!f) throw std::runtime_error(where + " > Truncated Cube");
  return v;
}

inline void MakeFolder(const std::string& path, const std::string& where) {
  struct stat st = {};
  if (stat(path.c_str(), &st) == -1 && mkdir(path.c_str(), 0755) == -1)
    throw std::runtime_error(where + " > Failed to Create Target Folder!");
}

// ---------------------------------------------------------------------------
// The GPU case shared by the phases
// ---------------------------------------------------------------------------
class GpuCase {
 public:
  explicit GpuCase(const tg_case& c) : c_(c) {
    Check("FlatChannelSolver::Configure", tg_create(&c_, &ctx_));
    int d[6];
    Check("FlatChannelSolver::Configure", tg_get_dims(ctx_, d));
    nxh_ = d[3];
    nyc_ = d[4];
  }
  ~GpuCase() {
    if (ctx_) tg_destroy(ctx_);
  }
  GpuCase(const GpuCase&) = delete;
  GpuCase& operator=(const GpuCase&) = delete;
  tg_ctx* ctx() const { return ctx_; }
  const tg_case& config() const { return c_; }
  int nz() const { return c_.nz; }
  int nyc() const { return nyc_; }
  int nxh() const { return nxh_; }
  size_t field() const { return (size_t)c_.nz * nyc_ * nxh_; }

 private:
  tg_case c_;
  tg_ctx* ctx_ = nullptr;
  int nxh_ = 0, nyc_ = 0;
};

// ---------------------------------------------------------------------------
// RK3TimeStepper: coefficients live in the library; the host keeps the step,
// time, dt, CFL and the forward / output flags (TimeStepper::Configure,
// Update for a fixed dt, Update2 for the adaptive dt).
// ---------------------------------------------------------------------------
class RK3TimeStepper {
 public:
  // TimeStepper::Configure (src/stepper_time.cc:215-246)
  void Configure(const tg_case& c, const RunControl& rc) {
    rc_ = rc;
    if (rc.output_based_on_step) {
      step_ = std::max(0, rc.startstep);
      dt_ = c.dt;
      time_ = step_ * dt_;
      isforward_ = step_ <= rc.maxstep;
    } else {
      step_ = 0;
      dt_ = rc.initial_time_step;
      time_ = rc.start_time_index > 0 ? rc.start_time_index * rc.output_interval : 0.0;
      output_time_index_ = rc.start_time_index;
      isforward_ = time_ <= rc.max_marching_time;
    }
  }
  // TimeStepper::Update (src/stepper_time.cc:72-113)
  void Update(double maxulen) {
    if (!isforward_) return;
    step_ += 1;
    time_ = time_ + dt_;
    isforward_ = step_ < rc_.maxstep;
    isoutput_ = step_ % rc_.writeinterval == 0;
    cfl_ = maxulen * dt_;
    if (cfl_ > rc_.maxcfl) {
      isforward_ = false;
      isoutput_ = true;
    }
  }
  // TimeStepper::Update2 (src/stepper_time.cc:117-208): time advances by the
  // previous dt, then dt is rescaled towards the CFL band and clipped to land
  // on the next output time.
  void Update2(double maxulen) {
    if (!isforward_) return;
    step_ += 1;
    time_ = time_ + dt_;
    isforward_ = time_ < rc_.max_marching_time;
    cfl_ = maxulen * dt_;
    if (cfl_ > 0) {
      const double top = rc_.cfl_adjust_scale[0], bot = rc_.cfl_adjust_scale[1];
      if (cfl_ > top * rc_.maxcfl) {
        dt_ = dt_ * top;
        while (maxulen * dt_ > top * rc_.maxcfl) dt_ = dt_ * top;
      } else if (cfl_ < bot * rc_.maxcfl) {
        dt_ = dt_ * 1.05;
      }
      if ((time_ + dt_) / rc_.output_interval - output_time_index_ - 1 >= 0) {
        const double dttmp = (output_time_index_ + 1) * rc_.output_interval - time_;
        dt_ = dttmp < rc_.initial_time_step / 100 ? dt_ / 20 : dttmp;
        output_time_index_ = output_time_index_ + 1;
        isoutput_ = true;
      } else {
        isoutput_ = false;
      }
    }
    if (cfl_ > rc_.maxcfl * 1.1 || dt_ < rc_.initial_time_step / 1000) {
      isforward_ = false;
      isoutput_ = true;
    }
  }
  void SetAlternationFlag() { alternation_ = !alternation_; }
  bool isForward() const { return isforward_; }
  bool isOutput() const { return isoutput_; }
  bool isOutputOnStep() const { return rc_.output_based_on_step != 0; }
  bool GetAlternationFlag() const { return alternation_; }
  int GetStep() const { return step_; }
  int GetOutputTimeIndex() const { return output_time_index_; }
  int GetStartIndex() const { return isOutputOnStep() ? rc_.startstep : rc_.start_time_index; }
  double GetTime() const { return time_; }
  double GetCfl() const { return cfl_; }
  double GetTimeStep() const { return dt_; }

 private:
  RunControl rc_;
  double dt_ = 0, time_ = 0, cfl_ = 0;
  int step_ = 0, output_time_index_ = 0;
  bool isforward_ = false, isoutput_ = false, alternation_ = false;
};

// ---------------------------------------------------------------------------
// Phases: Predict / Correct of one RK3 stage on the GPU; Save / Load of the
// restart variables (IO level one) in the reference's file layout.
// ---------------------------------------------------------------------------
class FlatCarrierPhase {
 public:
  explicit FlatCarrierPhase(GpuCase& g) : g_(g) {}
  void Predict(int stage) { Check("FlatCarrierPhase::Predict(int)", tg_carrier_predict(g_.ctx(), stage)); }
  void Correct(int stage) { Check("FlatCarrierPhase::Correct(int)", tg_carrier_correct(g_.ctx(), stage)); }
  std::vector<double> GetFeatureGlobal() const {
    std::vector<double> f(TG_NFEATURE);
    Check("Phase::GetFeatureGlobal", tg_features(g_.ctx(), f.data()));
    return f;
  }

 private:
  GpuCase& g_;
};

class FlatScalarPhase {
 public:
  explicit FlatScalarPhase(GpuCase& g) : g_(g) {}
  void Predict(int stage) { Check("FlatScalarPhase::Predict(int)", tg_scalar_predict(g_.ctx(), stage)); }
  void Correct(int stage) { Check("FlatScalarPhase::Correct(int)", tg_scalar_correct(g_.ctx(), stage)); }

 private:
  GpuCase& g_;
};

// Restart variables of both phases: phase_00_variable.dat (u, v, w as one
// cube of 3*Nxh slices, then p) and phase_01_variable.dat (the scalar).
class FlatVariables {
 public:
  explicit FlatVariables(GpuCase& g) : g_(g) {}
  void Load(const std::string& folder, int start_step) {
    const size_t n = g_.field();
    std::vector<std::complex<double>> uvw, p, phi;
    {
      std::ifstream f(folder + "phase_00_variable.dat", std::ios::binary);
      if (!f) throw std::runtime_error("FlatCarrierVariable::Load(int,ioctrl_t,string) > Can not Open " + folder + "phase_00_variable.dat");
      CheckLevel(f, "FlatCarrierVariable::Load(int,ioctrl_t,string)");
      uvw = ReadCube(f, g_.nz(), g_.nyc(), 3 * g_.nxh(), "FlatCarrierVariable::Load(int,ioctrl_t,string)");
      p = ReadCube(f, g_.nz(), g_.nyc(), g_.nxh(), "FlatCarrierVariable::Load(int,ioctrl_t,string)");
    }
    if (g_.config().nphase > 1) {
      std::ifstream f(folder + "phase_01_variable.dat", std::ios::binary);
      if (!f) throw std::runtime_error("FlatScalarVariable::Load(int,ioctrl_t,string) > Can not Open " + folder + "phase_01_variable.dat");
      CheckLevel(f, "FlatScalarVariable::Load(int,ioctrl_t,string)");
      phi = ReadCube(f, g_.nz(), g_.nyc(), g_.nxh(), "FlatScalarVariable::Load(int,ioctrl_t,string)");
    }
    (void)n;
    Check("FlatCarrierVariable::Load(int,ioctrl_t,string)",
          tg_upload_state(g_.ctx(), reinterpret_cast<const double*>(uvw.data()),
                          reinterpret_cast<const double*>(p.data()),
                          phi.empty() ? nullptr : reinterpret_cast<const double*>(phi.data()), start_step));
  }
  void Save(const std::string& folder) {
    const size_t n = g_.field();
    std::vector<std::complex<double>> uvw(3 * n), p(n), phi(g_.config().nphase > 1 ? n : 0);
    Check("FlatCarrierVariable::Save(int,ioctrl_t,string)",
          tg_download_state(g_.ctx(), reinterpret_cast<double*>(uvw.data()), reinterpret_cast<double*>(p.data()),
                            phi.empty() ? nullptr : reinterpret_cast<double*>(phi.data())));
    MakeFolder(folder, "FlatCarrierVariable::Save(int,ioctrl_t,string)");
    {
      std::ofstream f(folder + "phase_00_variable.dat", std::ios::binary);
      f << "IOControlLevelOne\n";
      WriteCube(f, uvw, g_.nz(), g_.nyc(), 3 * g_.nxh());
      WriteCube(f, p, g_.nz(), g_.nyc(), g_.nxh());
    }
    if (!phi.empty()) {
      std::ofstream f(folder + "phase_01_variable.dat", std::ios::binary);
      f << "IOControlLevelOne\n";
      WriteCube(f, phi, g_.nz(), g_.nyc(), g_.nxh());
    }
  }

 private:
  static void CheckLevel(std::istream& f, const std::string& where) {
    std::string level;
    std::getline(f, level);
    if (level != "IOControlLevelOne") throw std::runtime_error(where + " > Wrong Request of IO Level One!");
  }
  GpuCase& g_;
};

// ---------------------------------------------------------------------------
// FlatChannelSolver: Configure from the .ini, Execute the step loop
// ---------------------------------------------------------------------------
class FlatChannelSolver {
 public:
  // argv[1]: configuration file (default configuration.ini), argv[2]: log
  // file (default logcomputation); --mixed selects mixed precision, as does
  // gpu_precision = Mixed in the file's [System] section.
  FlatChannelSolver(int argc, char** argv) {
    std::vector<std::string> pos;
    for (int i = 1; i < argc; ++i) {
      const std::string a = argv[i];
      if (a == "--mixed") mixed_flag_ = true;
      else pos.push_back(a);
    }
    if (pos.size() > 0) config_ = pos[0];
    if (pos.size() > 1) logname_ = pos[1];
    const size_t slash = config_.find_last_of('/');
    directory_ = slash == std::string::npos ? "./" : config_.substr(0, slash + 1);
  }
  void Configure() {
    ini_.Load(config_);
    precision_ = TG_PREC_FP64;
    if (ini_.HasKey("System", "gpu_precision")) {
      const std::string pr = Upper(ini_.GetValueString("System", "gpu_precision"));
      if (pr == "MIXED") precision_ = TG_PREC_MIXED;
      else if (pr != "FP64") throw std::runtime_error("FlatChannelSolver::Configure > gpu_precision must be FP64 or Mixed");
    }
    if (mixed_flag_) precision_ = TG_PREC_MIXED;
    const tg_case c = CaseFromIni(ini_, rc_, precision_);
    gpu_.reset(new GpuCase(c));
    carrier_.reset(new FlatCarrierPhase(*gpu_));
    if (c.nphase > 1) scalar_.reset(new FlatScalarPhase(*gpu_));
    variables_.reset(new FlatVariables(*gpu_));
    tstepper_.Configure(c, rc_);
    // FlatCarrierVariable::Configure (src/variable_carrier_flat.cc:386-401)
    const int inputindex = tstepper_.GetStartIndex();
    if (inputindex < 0) throw std::runtime_error("FlatCarrierVariable::Configure > A Restart State is Required (start index < 0)");
    variables_->Load(directory_ + std::to_string((long long)inputindex) + "/", tstepper_.GetStep());
    configured_ = true;
  }
  bool isConfigured() const { return configured_; }
  const RK3TimeStepper& TimeStepper() const { return tstepper_; }

  // FlatChannelSolver::Execute (src/solver_channel_flat.cc:199-293)
  void Execute() {
    if (!configured_) throw std::runtime_error("FlatChannelSolver::Execute > Not Configured!");
    std::ofstream log(directory_ + logname_, std::ios::app);
    std::vector<double>& feature = feature_;
    feature = carrier_->GetFeatureGlobal();
    while (tstepper_.isForward()) {
      // a CFL above the limit (or the last step) clears the forward flag; the
      // step is still taken and, with the output flag, written for record.
      // With the adaptive dt, tg_set_time re-assembles the solves for the new
      // dt (FlatCarrierPhase::Update / FlatScalarPhase::Update).
      if (tstepper_.isOutputOnStep())
        tstepper_.Update(feature[19]);
      else
        tstepper_.Update2(feature[19]);
      Check("TimeStepper::Update", tg_set_time(gpu_->ctx(), tstepper_.GetStep(), tstepper_.GetTime(),
                                                tstepper_.GetTimeStep(), tstepper_.GetAlternationFlag() ? 1 : 0));
      for (int stage = 0; stage < 3; ++stage) {
        carrier_->Predict(stage);
        carrier_->Correct(stage);
        if (scalar_) {
          scalar_->Predict(stage);
          scalar_->Correct(stage);
        }
      }
      tstepper_.SetAlternationFlag();
      feature = carrier_->GetFeatureGlobal();
      if (tstepper_.isOutput()) {
        const int index = tstepper_.isOutputOnStep() ? tstepper_.GetStep() : tstepper_.GetOutputTimeIndex();
        variables_->Save(directory_ + std::to_string((long long)index) + "/");
      }
      std::ostringstream line;
      PrintLogBody(line, feature);
      std::cout << line.str();
      log << line.str();
    }
    Check("FlatChannelSolver::Execute", tg_synchronize(gpu_->ctx()));
  }

  // Case summary written before the first log line: grid, precision, time
  // stepping and the physical parameters (the reference prints its component
  // objects there, src/solver_channel_flat.cc:340-366).
  void PrintLogHead(std::ostream& s) const {
    const std::string sep(80, '*');
    s << sep << "\n";
    if (gpu_) {
      const tg_case& c = gpu_->config();
      s << std::setw(30) << std::right << "FlatChannelSolver > " << "grid " << c.nx << " x " << c.ny << " x " << c.nz
        << ", phases " << c.nphase << ", precision " << (c.precision == TG_PREC_MIXED ? "Mixed" : "FP64") << "\n";
      s << std::setw(30) << std::right << "RK3TimeStepper > " << std::setprecision(10) << "dt " << tstepper_.GetTimeStep()
        << ", start step " << tstepper_.GetStep() << ", max step " << rc_.maxstep << ", max cfl " << rc_.maxcfl << "\n";
      s << std::setw(30) << std::right << "FlatCarrierPhase > " << "Re " << c.reynolds << ", force type " << c.force_type
        << "\n";
      if (c.nphase > 1)
        s << std::setw(30) << std::right << "FlatScalarPhase > " << "Sc " << c.schmidt << ", Ws " << c.settling
          << ", boundary " << (c.scalar_bc ? "ErosionDeposition" : "ZeroFlux") << "\n";
    }
    s << sep << "\n";
  }
  // The last step's log line (the features read after that step).
  void PrintLogBody(std::ostream& s) const { PrintLogBody(s, feature_); }
  const std::vector<double>& Features() const { return feature_; }

  // FlatChannelSolver::PrintLogBody (src/solver_channel_flat.cc:372-414)
  void PrintLogBody(std::ostream& s, const std::vector<double>& f) const {
    s << std::setw(12) << tstepper_.GetStep() << std::setw(16) << std::setprecision(10) << tstepper_.GetTime()
      << std::setw(12) << std::setprecision(6) << tstepper_.GetCfl();
    for (int i : {0, 1, 2, 3, 4, 5, 6, 7, 8, 10, 11, 12, 13, 14, 15, 21, 22, 23, 24, 25, 28, 29})
      s << std::setw(12) << f[i];
    s << std::endl;
  }

 private:
  std::string config_ = "configuration.ini", logname_ = "logcomputation", directory_ = "./";
  int precision_ = TG_PREC_FP64;
  bool mixed_flag_ = false;
  bool configured_ = false;
  std::vector<double> feature_ = std::vector<double>(TG_NFEATURE, 0.0);
  IniFile ini_;
  RunControl rc_;
  RK3TimeStepper tstepper_;
  std::unique_ptr<GpuCase> gpu_;
  std::unique_ptr<FlatCarrierPhase> carrier_;
  std::unique_ptr<FlatScalarPhase> scalar_;
  std::unique_ptr<FlatVariables> variables_;
};

// ---------------------------------------------------------------------------
// FlatChannelPostprocessor: swirling strength of the saved states
// [PostProcessor] work_index_range = first last; writes
// <index>/phase_00_vortex.dat (Armadillo binary real cube, Nx x Ny x Nz)
// ---------------------------------------------------------------------------
class FlatChannelPostprocessor {
 public:
  FlatChannelPostprocessor(int argc, char** argv) {
    for (int i = 1; i < argc; ++i) {
      const std::string a = argv[i];
      if (a.rfind("--", 0) != 0) {
        config_ = a;
        break;
      }
    }
    const size_t slash = config_.find_last_of('/');
    directory_ = slash == std::string::npos ? "./" : config_.substr(0, slash + 1);
  }
  void Configure() {
    ini_.Load(config_);
    RunControl rc;
    gpu_.reset(new GpuCase(CaseFromIni(ini_, rc)));
    variables_.reset(new FlatVariables(*gpu_));
    range_ = ini_.GetVectorInt("PostProcessor", "work_index_range");
    if (range_.size() != 2) throw std::runtime_error("FlatChannelPostprocessor::Configure > work_index_range needs 2 values");
  }
  void Execute() {
    const tg_case& c = gpu_->config();
    std::vector<double> vortex((size_t)c.nx * c.ny * c.nz);
    for (int index = range_[0]; index <= range_[1]; ++index) {
      const std::string path = directory_ + std::to_string((long long)index) + "/";
      variables_->Load(path, 0);
      Check("FlatChannelPostprocessor::Execute", tg_swirling_strength(gpu_->ctx(), vortex.data()));
      std::ofstream f(path + "phase_00_vortex.dat", std::ios::binary);
      if (!f) throw std::runtime_error("FlatChannelPostprocessor::Execute > Can not Open " + path + "phase_00_vortex.dat");
      f << "ARMA_CUB_BIN_FN008\n" << c.nx << " " << c.ny << " " << c.nz << "\n";
      f.write(reinterpret_cast<const char*>(vortex.data()), (std::streamsize)(vortex.size() * sizeof(double)));
      std::cout << std::setw(12) << index << std::endl;
    }
  }

 private:
  std::string config_ = "configuration.ini", directory_ = "./";
  IniFile ini_;
  std::vector<int> range_;
  std::unique_ptr<GpuCase> gpu_;
  std::unique_ptr<FlatVariables> variables_;
};

}  // namespace turbid
