// The reference's main program (main/channelflat.cc) with the GPU plugin
// classes: reads configuration.ini (or argv[1]) and the restart files of
// task_start_step, runs the RK3 steps on the GPU, writes the restart files
// every result_write_interval steps and one log line per step.
//
//   channelflat_gpu [configuration.ini [logcomputation]] [--mixed]
//   channelflat_gpu --parse-only configuration.ini    (case parameters as JSON, no GPU)
//   channelflat_gpu --postprocess [configuration.ini]  (swirling strength of the states
//       of [PostProcessor] work_index_range, written as <index>/phase_00_vortex.dat)
//   channelflat_gpu --time-only configuration.ini L1 L2 ...
//       (the time stepper alone for the given per-step maximum velocity/length
//        values: one JSON line per step with step, time, dt, cfl, flags; no GPU)
#include <iostream>
#include <string>

#include "turbid_plugin.hpp"

namespace {
void PrintCaseJson(const tg_case& c, const turbid::RunControl& rc) {
  auto vec = [](const double* v, int n) {
    std::ostringstream s;
    s << "[";
    for (int i = 0; i < n; ++i) s << (i ? ", " : "") << std::setprecision(17) << v[i];
    s << "]";
    return s.str();
  };
  std::ostringstream s;
  s << std::setprecision(17) << "{\"nx\": " << c.nx << ", \"ny\": " << c.ny << ", \"nz\": " << c.nz
    << ", \"lx\": " << c.lx << ", \"ly\": " << c.ly << ", \"nphase\": " << c.nphase << ", \"mapping\": " << c.mapping
    << ", \"mapping_coef\": " << c.mapping_coef << ", \"slope\": " << c.slope
    << ", \"slope_direction\": " << c.slope_direction << ", \"dt\": " << c.dt
    << ", \"output_based_on_step\": " << c.output_based_on_step << ", \"reynolds\": " << c.reynolds
    << ", \"froude\": " << c.froude << ", \"averaged_concentration\": " << c.averaged_concentration
    << ", \"specific_gravity\": " << c.specific_gravity << ", \"affected_by_scalar\": " << c.affected_by_scalar
    << ", \"bc_u\": " << vec(c.bc_u, 5) << ", \"bc_v\": " << vec(c.bc_v, 5) << ", \"bc_w\": " << vec(c.bc_w, 5)
    << ", \"bc_p\": " << vec(c.bc_p, 5) << ", \"force_type\": " << c.force_type << ", \"force_direction\": ["
    << c.force_direction[0] << ", " << c.force_direction[1] << "], \"force_amplitude\": " << vec(c.force_amplitude, 2)
    << ", \"schmidt\": " << c.schmidt << ", \"settling\": " << c.settling << ", \"erosion_rate\": " << c.erosion_rate
    << ", \"critical_shear\": " << c.critical_shear << ", \"scalar_bc\": " << c.scalar_bc
    << ", \"maxcfl\": " << rc.maxcfl << ", \"maxstep\": " << rc.maxstep << ", \"writeinterval\": " << rc.writeinterval
    << ", \"startstep\": " << rc.startstep << ", \"max_marching_time\": " << rc.max_marching_time
    << ", \"output_interval\": " << rc.output_interval << ", \"initial_time_step\": " << rc.initial_time_step
    << ", \"start_time_index\": " << rc.start_time_index << ", \"cfl_adjust_scale\": "
    << vec(rc.cfl_adjust_scale, 2) << "}";
  std::cout << s.str() << std::endl;
}
}  // namespace

int main(int argc, char** argv) {
  try {
    if (argc > 2 && std::string(argv[1]) == "--parse-only") {
      turbid::IniFile ini;
      ini.Load(argv[2]);
      turbid::RunControl rc;
      PrintCaseJson(turbid::CaseFromIni(ini, rc), rc);
      return 0;
    }
    if (argc > 2 && std::string(argv[1]) == "--time-only") {
      turbid::IniFile ini;
      ini.Load(argv[2]);
      turbid::RunControl rc;
      const tg_case c = turbid::CaseFromIni(ini, rc);
      turbid::RK3TimeStepper ts;
      ts.Configure(c, rc);
      for (int i = 3; i < argc && ts.isForward(); ++i) {
        const double maxulen = std::atof(argv[i]);
        if (ts.isOutputOnStep()) ts.Update(maxulen);
        else ts.Update2(maxulen);
        std::cout << std::setprecision(17) << "{\"step\": " << ts.GetStep() << ", \"time\": " << ts.GetTime()
                  << ", \"dt\": " << ts.GetTimeStep() << ", \"cfl\": " << ts.GetCfl()
                  << ", \"forward\": " << (ts.isForward() ? 1 : 0) << ", \"output\": " << (ts.isOutput() ? 1 : 0)
                  << ", \"output_index\": " << ts.GetOutputTimeIndex() << "}" << std::endl;
      }
      return 0;
    }
    if (argc > 1 && std::string(argv[1]) == "--postprocess") {
      turbid::FlatChannelPostprocessor post(argc, argv);
      post.Configure();
      post.Execute();
      return 0;
    }
    turbid::FlatChannelSolver solver(argc, argv);
    solver.Configure();
    solver.Execute();
  } catch (std::runtime_error& err) {
    std::cout << err.what() << std::endl;
    return 1;
  }
  return 0;
}
