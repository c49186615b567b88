// ndg_internal.h -- context hooks the serving loop (ndg_server.cpp) uses
// beside the public ABI; not exported from the library's C interface.
#pragma once
#include <vector>

#include "../../include/ndyn_gpu.h"

namespace ndg_internal {

// dynamics prologue (skin, MCELL, list capacity, one list build) for the
// given systems only; the others keep their lists and state
int setup_systems(ndg_ctx *c, const std::vector<int> &ids);
// give one system a run of nsteps that starts with its lists just built
int arm_built(ndg_ctx *c, int sys, int nsteps);
// one block of up to K steps for every system with steps left in its run;
// thermo records go to cb
int run_block(ndg_ctx *c, int K, ndg_thermo_cb cb, void *user);
// apply one system's pending velocity scales (the end of its run)
int flush_system(ndg_ctx *c, int sys);
// step-block graphs captured so far
int graph_captures(ndg_ctx *c);
// error bits recorded on one system (E_* of ndg_common.h), then cleared
int take_system_error(ndg_ctx *c, int sys, int *err);
// room at the end of the atom arena for `atoms` more atoms of systems about
// to be added (one growth for a whole admission batch)
int reserve_atoms(ndg_ctx *c, long long atoms);

}  // namespace ndg_internal
