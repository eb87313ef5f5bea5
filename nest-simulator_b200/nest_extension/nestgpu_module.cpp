/*
 * nestgpu_module.cpp -- the NEST extension module (NESTExtensionInterface,
 * nestkernel/nest_extension_interface.h) that registers the gpu_engine node
 * model (register_node_model, nestkernel/nest.h:101).
 *
 * Two ways in:
 *  - nest.Install("nestgpu_module") where NEST was built with libltdl: the
 *    ModuleManager looks up the symbol `module` and calls its initialize()
 *    (nestkernel/module_manager.cpp:112-181);
 *  - without libltdl: load the library with RTLD_GLOBAL after `import nest`
 *    and call nestgpu_init() (ctypes).
 */
#include "nest_extension_interface.h"

#include "gpu_engine.h"

namespace nestgpu
{

class NestGpuModule : public nest::NESTExtensionInterface
{
public:
  ~NestGpuModule() override
  {
  }

  void
  initialize() override
  {
    nest::register_node_model< gpu_engine >( "gpu_engine" );
  }
};

}  // namespace nestgpu

// the instance the ModuleManager finds by the unmangled name `module`
extern "C"
{
  nestgpu::NestGpuModule module;

  int
  nestgpu_init( void )
  {
    try
    {
      module.initialize();
    }
    catch ( ... )
    {
      return -1;
    }
    return 0;
  }
}
