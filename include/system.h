/* system.h -- the System base class of the reference's solver layer
 * (yueliangyi/TURBID src/system.h:33-95) as the GPU build ships it.
 *
 * main/channelflat.cc sees this class through solver_channel_flat.h: it
 * constructs a FlatChannelSolver from (argc, argv), calls Configure(),
 * isConfigured() and Execute(), and catches std::runtime_error.  The GPU build
 * keeps those names, signatures and the argv meaning (argv[1] configuration
 * file, default "configuration.ini"; argv[2] log file, default
 * "logcomputation"; src/system.cc:19-37).  The MPI group, the domain
 * decomposition and the component objects of the reference's System are not
 * part of this interface: the whole case lives in one GPU context, held by the
 * solver (libpseudospectral.so over libturbid_gpu.so).
 */
#ifndef TURBID_PS_SYSTEM_H_
#define TURBID_PS_SYSTEM_H_

#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>

namespace yueliangyi {
namespace pseudospectral {
namespace leveltwo {

class System {
 public:
  System(int& argc, char**& argv);
  virtual ~System(void) {}

  bool isConfigured(void) { return isconfigured_; }

  virtual bool Configure(void) = 0;
  virtual bool Execute(void) = 0;

  virtual void Print(std::ostringstream& stream) const;
  virtual void PrintLogHead(std::ostringstream& stream) const = 0;
  virtual void PrintLogBody(std::ostringstream& stream) const = 0;

 protected:
  System(const System& other) = delete;

  std::string file_configuration_ = "configuration.ini";
  std::string file_log_ = "logcomputation";
  bool isconfigured_ = false;
};

}  // namespace leveltwo
}  // namespace pseudospectral
}  // namespace yueliangyi

#endif  // TURBID_PS_SYSTEM_H_
