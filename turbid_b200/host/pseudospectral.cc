// libpseudospectral.so of the GPU build: the reference's solver-layer classes
// System and FlatChannelSolver (include/system.h, include/solver_channel_flat.h)
// over the plugin classes of turbid_plugin.hpp, which call libturbid_gpu.so.
// The reference's main/channelflat.cc links against this library unchanged
// (-lpseudospectral, as in its Makefile:30,83-86).
#include <fstream>
#include <memory>

#include "solver_channel_flat.h"
#include "turbid_plugin.hpp"

namespace yueliangyi {
namespace pseudospectral {
namespace leveltwo {

// System::System (src/system.cc:19-37): argv[1] configuration file, argv[2]
// log file.
System::System(int& argc, char**& argv) {
  if (argc > 1) file_configuration_ = std::string(argv[1]);
  if (argc > 2) file_log_ = std::string(argv[2]);
}

void System::Print(std::ostringstream& stream) const {
  stream << "configuration " << file_configuration_ << ", log " << file_log_;
}

struct FlatChannelSolver::Impl {
  std::unique_ptr<turbid::FlatChannelSolver> solver;
  std::string directory = "./";
};

// FlatChannelSolver::FlatChannelSolver (src/solver_channel_flat.cc:31-120):
// the case file is read by Configure below (the GPU context is created there).
FlatChannelSolver::FlatChannelSolver(int& argc, char**& argv) : System(argc, argv), impl_(new Impl) {
  impl_->solver.reset(new turbid::FlatChannelSolver(argc, argv));
  const size_t slash = file_configuration_.find_last_of('/');
  if (slash != std::string::npos) impl_->directory = file_configuration_.substr(0, slash + 1);
}

FlatChannelSolver::~FlatChannelSolver(void) { delete impl_; }

// FlatChannelSolver::Configure (src/solver_channel_flat.cc:148-172): case
// parameters, operators and decompositions on the GPU, restart state of
// task_start_step.
bool FlatChannelSolver::Configure(void) {
  impl_->solver->Configure();
  isconfigured_ = impl_->solver->isConfigured();
  return isconfigured_;
}

// FlatChannelSolver::Execute (src/solver_channel_flat.cc:179-313): the log
// head, then the step loop with its log lines and restart files.
bool FlatChannelSolver::Execute(void) {
  if (!isconfigured_) throw std::runtime_error(name_ + "Execute > Not Configured!");
  std::ostringstream head;
  PrintLogHead(head);
  std::cout << head.str();
  {
    std::ofstream log(impl_->directory + file_log_, std::ios::app);
    log << head.str();
  }
  impl_->solver->Execute();
  return true;
}

void FlatChannelSolver::Print(std::ostringstream& stream) const {
  stream << "FlatChannelSolver > ";
  System::Print(stream);
  stream << std::endl;
}

void FlatChannelSolver::PrintLogHead(std::ostringstream& stream) const {
  impl_->solver->PrintLogHead(stream);
}

// One log line of the last step (src/solver_channel_flat.cc:372-414).
void FlatChannelSolver::PrintLogBody(std::ostringstream& stream) const {
  impl_->solver->PrintLogBody(stream);
}

}  // namespace leveltwo
}  // namespace pseudospectral
}  // namespace yueliangyi
