/* solver_channel_flat.h -- FlatChannelSolver of the reference's solver layer
 * (yueliangyi/TURBID src/solver_channel_flat.h:13-27) as the GPU build ships
 * it, so that the reference's main/channelflat.cc compiles unchanged:
 *
 *   g++ -I<repo>/include main/channelflat.cc -L<repo>/turbid_b200 \
 *       -lpseudospectral -Wl,-rpath,<repo>/turbid_b200
 *
 * libpseudospectral.so implements the class over the C ABI of libturbid_gpu.so
 * (the plugin classes of turbid_plugin.hpp): Configure() reads the case file
 * and the restart state of task_start_step (src/solver_channel_flat.cc:
 * 148-172), Execute() runs the RK3 steps on the GPU, writes the restart files
 * every result_write_interval steps and one log line per step
 * (src/solver_channel_flat.cc:179-313).  Errors are std::runtime_error with
 * "Class::Method > message" text, as in the reference.
 *
 * Precision: FP64 unless the case file's [System] section sets
 * gpu_precision = Mixed, or the command line carries --mixed after the file
 * names (the reference reads argv[1] and argv[2] only and ignores the rest).
 */
#ifndef TURBID_PS_SOLVER_CHANNEL_FLAT_H_
#define TURBID_PS_SOLVER_CHANNEL_FLAT_H_

#include "system.h"

namespace yueliangyi {
namespace pseudospectral {
namespace leveltwo {

class FlatChannelSolver : public System {
 public:
  FlatChannelSolver(int& argc, char**& argv);
  ~FlatChannelSolver(void);

  bool Configure(void);
  bool Execute(void);

  void Print(std::ostringstream& stream) const;
  void PrintLogHead(std::ostringstream& stream) const;
  void PrintLogBody(std::ostringstream& stream) const;

 protected:
  std::string name_ = "FlatChannelSolver::";

 private:
  struct Impl;
  Impl* impl_;
};

}  // namespace leveltwo
}  // namespace pseudospectral
}  // namespace yueliangyi

#endif  // TURBID_PS_SOLVER_CHANNEL_FLAT_H_
