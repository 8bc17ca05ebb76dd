// integrator_group.h -- the plain FP64 GPU path (integrator_group.cu): one
// BDF integration per group of reactors with a shared step size, order and
// WRMS norm, driven from the host kernel by kernel, as the reference's GPU
// branch of the cfd_plugin integrates a batch with one CVODE instance.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "integrator.h"

namespace zrk {

struct GroupCounters {
  long groups = 0, group_steps = 0, group_newton = 0, launches = 0, syncs = 0;
  long first_fail = 0;  // status of the first group whose attempts all failed
};

// Doubles of device workspace per reactor of a group (the reactor's BDF
// vectors, history, Jacobian and Newton-matrix inverse).
size_t group_slot_doubles(const DevMech &m);
// Group sizes for n reactors and at most group_max per group, the last two
// groups split evenly (zerork_reactor_manager.cpp:933-940).
int group_sizes(int n, int group_max, std::vector<int> &sizes);
// Integrate a.n_reactors reactors (order_dev: reactor indices in group
// order) group by group.  slots: group_max * group_slot_doubles doubles;
// part_dev / part_host (pinned): group_max * 6 doubles each.  Per-reactor
// statistics go to a.stats (every reactor of a group gets the group's
// counters and status).  a.state / a.lu / a.order / a.queue_head unused.
cudaError_t integrate_group(const DevMech &m, const IntegOpts &o, const IntegArgs &a, const int *order_dev,
                            int group_max, int threads, double *slots, double *part_dev,
                            double *part_host, cudaStream_t stream, GroupCounters *gc);

}  // namespace zrk
