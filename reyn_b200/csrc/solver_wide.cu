// The step with the neighbour passes compiled for blocks of up to 512
// threads (block sizes 256 and 512, chosen by reyn_params.block_size or the
// autotuner); a separate translation unit so that the two instantiations
// of the passes build in parallel.
#include "passes.cuh"

namespace reyn {

void solver_step_wide(reyn_solver& sv, reyn_particles& st, const Grid& grid,
    const reyn_boundary* bdy, float dt, cudaStream_t s, const float* bmin, const float* bmax)
{
    solver_step_t<NBR_MAX_THREADS>(sv, st, grid, bdy, dt, s, bmin, bmax);
}

} // namespace reyn
