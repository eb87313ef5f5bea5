/*
 * gpu_engine.h -- a NEST node that runs a population of the reference's own
 * neurons on the B200 engine (include/nestgpu.h).
 *
 * The user builds the network with PyNEST as usual (nest.Create, nest.Connect,
 * poisson_generator drive, spike_recorder), then creates one gpu_engine and
 * points it at a contiguous range of neurons:
 *
 *   pop = nest.Create("iaf_psc_exp", 12500, ...)
 *   ...
 *   eng = nest.Create("gpu_engine", params={"first_node_id": pop[0].global_id,
 *                                          "n_nodes": len(pop)})
 *   nest.Simulate(1000.0)
 *
 * At the first Prepare (pre_run_hook) the engine reads each neuron's
 * parameters and state (Node::get_status_base), the static_synapse
 * connections among them and from poisson_generators into them (the
 * reference's own GetConnections: ConnectionManager::get_connections,
 * nestkernel/connection_manager.h:250, and get_synapse_status :219), uploads
 * them, and freezes the neurons, so SimulationManager::update_ skips them
 * (the frozen test at nestkernel/simulation_manager.cpp:1067).  Every slice
 * its update(origin, from, to) (nestkernel/node.h:297) enqueues the same
 * steps on the GPU (ng_update) without waiting.  At the end of each Run
 * (post_run_cleanup) it drains the spikes and hands each one to the
 * recording devices connected to its neuron through
 * ConnectionManager::send_to_devices (nestkernel/connection_manager.h:312)
 * -- the path EventDeliveryManager::send takes for a neuron's spike
 * (nestkernel/event_delivery_manager_impl.h:60-84) -- so spike_recorder
 * windows and backends are the reference's own; the neurons' state is
 * written back, so GetStatus on them reads the GPU's values.
 *
 * Supported: one model per engine among iaf_psc_delta, iaf_psc_exp,
 * iaf_psc_alpha and aeif_cond_alpha; static_synapse connections, and
 * stdp_pl_synapse_hom connections (or copies of it) among the population's
 * neurons with one set of common properties -- their weights are written
 * back after each Run (sync_weights) and the neurons' tau_minus is read;
 * one poisson_generator rate, weight and delay per neuron; local_num_threads
 * = 1 and one MPI process (the engine owns the whole population); the
 * engine takes the population over at time 0.  Anything else raises
 * BadProperty at Prepare.
 */
#ifndef NESTGPU_GPU_ENGINE_H
#define NESTGPU_GPU_ENGINE_H

#include <string>
#include <vector>

#include "connection_id.h"
#include "nest_time.h"
#include "node.h"

#include "../../include/nestgpu.h"

namespace nestgpu
{

class gpu_engine : public nest::Node
{
public:
  gpu_engine();
  gpu_engine( const gpu_engine& );
  ~gpu_engine() override;

  // one instance per process, not a neuron: no proxies, no incoming events
  bool
  has_proxies() const override
  {
    return false;
  }
  bool
  one_node_per_process() const override
  {
    return true;
  }
  bool
  local_receiver() const override
  {
    return false;
  }

  void get_status( Dictionary& ) const override;
  void set_status( const Dictionary& ) override;

  void pre_run_hook() override;
  void update( nest::Time const& origin, const long from, const long to ) override;
  void post_run_cleanup() override;
  void finalize() override;

private:
  void init_buffers_() override;

  void build_();         // read the population and its connections, create and fill the engine
  void drain_and_route_();  // spikes to the recording devices, state back to the neurons
  void release_();

  struct Parameters_
  {
    long first_node_id = 0;
    long n_nodes = 0;
    long device = 0;
    std::string precision = "fp64";
    long seed = 1;  // key of the Philox stream that replaces the poisson_generators' draws
    bool sync_weights = true;  // write the plastic weights back into NEST after each Run
  } P_;

  ng_engine* eng_ = nullptr;
  int model_ = -1;        // NG_IAF_PSC_DELTA / NG_IAF_PSC_EXP / NG_AEIF_COND_ALPHA
  double E_L_ = 0.0;      // per-population offset of the relative voltages (iaf models)
  std::vector< double > E_L_per_node_;
  std::vector< nest::ConnectionID > pl_conns_;  // the stdp_pl_synapse_hom connections, as NEST listed them
  std::vector< int64_t > pl_pos_;               // ... and each one's index in the engine's plastic CSR
  std::vector< int32_t > src_buf_;
  std::vector< int64_t > stamp_buf_;
  long long routed_ = 0;  // spikes handed to recording devices
};

}  // namespace nestgpu

#endif
