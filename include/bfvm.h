/* bfvm.h -- C ABI of the B200-native BioFVM transport path (libbfvm.so).
 *
 * One bfvm_solver holds the device state of one BioFVM Microenvironment: the
 * density field (resident in HBM, layout [voxel][substrate], voxel
 * n = (k*ny + j)*nx + i, the reference's own logical order), the Thomas
 * coefficients, the bulk source/sink table, the Dirichlet nodes and the
 * agents' secretion/uptake constants.  Host pointers in every signature are
 * plain host memory; nothing here takes or returns a torch type.
 *
 * Each entry point names the reference interface it replaces (file:line in
 * the BioFVM 1.0.4 source tree).  Every call returns 0 on success or a
 * BFVM_ERR_* code; bfvm_last_error() gives a message for the calling thread.
 * Work is enqueued on the solver's CUDA stream; calls that return host data
 * synchronise that stream.  Calls on one solver must not race from several
 * host threads. */
#ifndef BFVM_H
#define BFVM_H

#include <stdint.h>

#if defined(__GNUC__)
#define BFVM_API __attribute__((visibility("default")))
#else
#define BFVM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define BFVM_OK 0
#define BFVM_ERR_ARG 1     /* bad argument (size, index, pointer)            */
#define BFVM_ERR_CUDA 2    /* a CUDA runtime call failed                      */
#define BFVM_ERR_STATE 3   /* call not valid in the current state             */
#define BFVM_ERR_NOMEM 4   /* device or host allocation failed                */
#define BFVM_ERR_MESH 5    /* LOD_3D needs a uniform Cartesian mesh           */

/* step flags for bfvm_step: the three simulate_* calls of one step */
#define BFVM_STEP_BULK 1
#define BFVM_STEP_CELLS 2
#define BFVM_STEP_DIFFUSION 4
#define BFVM_STEP_ALL 7

/* precision of the density field and the sweeps */
#define BFVM_FP64 64
#define BFVM_FP32 32
/* FP32 field (half the memory traffic of FP64) swept in FP64 arithmetic with
 * FP64 coefficients: only the stored field is rounded to FP32 */
#define BFVM_FP32_FP64MATH 3264

typedef struct bfvm_solver bfvm_solver;

/* Message of the last failed call on this host thread ("" if none). */
BFVM_API const char* bfvm_last_error(void);
BFVM_API int bfvm_version(void);

/* Microenvironment::Microenvironment() (BioFVM_microenvironment.cpp:88-139):
 * a 1x1x1 mesh with one density, D = decay = 0, LOD_3D solver selected. */
BFVM_API int bfvm_create(bfvm_solver** out, int device);
BFVM_API int bfvm_destroy(bfvm_solver* m);

/* Microenvironment::resize_space(x0,x1,y0,y1,z0,z1,dx,dy,dz)
 * (BioFVM_microenvironment.cpp:267-285 -> Cartesian_Mesh::resize,
 * BioFVM_mesh.cpp:796-922): node counts ceil(1e-16 + L/d).  Densities are
 * reset to zero, Dirichlet nodes, bulk table and agents are cleared. */
BFVM_API int bfvm_resize_space(bfvm_solver* m, double x0, double x1, double y0, double y1, double z0,
                      double z1, double dx, double dy, double dz);
/* Microenvironment::resize_space(x0,...,z1, nx, ny, nz)
 * (BioFVM_microenvironment.cpp:246-265 -> BioFVM_mesh.cpp:663-794). */
BFVM_API int bfvm_resize_space_nodes(bfvm_solver* m, double x0, double x1, double y0, double y1,
                            double z0, double z1, int nx, int ny, int nz);
/* Restores a mesh exactly as bfvm_get_mesh describes it (nxyz[3], geom[10],
 * uniform flag), e.g. for a copy of a Microenvironment or a restart; no
 * counterpart call in the reference, whose Cartesian_Mesh members are public.
 * Densities are reset to zero and the lists cleared, as by a resize. */
BFVM_API int bfvm_set_mesh(bfvm_solver* m, const int* nxyz, const double* geom, int uniform);
/* nxyz[3] node counts; geom[10] = dx, dy, dz, dV, bounding box
 * (xmin, ymin, zmin, xmax, ymax, zmax); flags[2] = uniform_mesh, S. */
BFVM_API int bfvm_get_mesh(bfvm_solver* m, int* nxyz, double* geom, int* flags);

/* Microenvironment::resize_densities (BioFVM_microenvironment.cpp:292-323):
 * S densities, all zero, D = decay = 0. */
BFVM_API int bfvm_resize_densities(bfvm_solver* m, int num_densities);
/* Microenvironment::add_density(name, units, D, decay)
 * (BioFVM_microenvironment.cpp:404-441): appends one zero density.  After
 * the Thomas setup (the first step) the coefficient tables are rebuilt for
 * the new count from the setup's dt and coefficients: the existing densities
 * keep theirs, the new one gets its own (the reference keeps tables sized for
 * the old count there, and its next solve reads past them). */
BFVM_API int bfvm_add_density(bfvm_solver* m, double diffusion_coefficient, double decay_rate);
/* Microenvironment::set_density(index, name, units, D, decay)
 * (BioFVM_microenvironment.cpp:450-458) and the public
 * diffusion_coefficients / decay_rates vectors (BioFVM_microenvironment.h:118-119).
 * Read by the next Thomas set-up (see bfvm_reset_diffusion_setup). */
BFVM_API int bfvm_set_density_coefficients(bfvm_solver* m, int index, double diffusion_coefficient,
                                  double decay_rate);
BFVM_API int bfvm_get_num_densities(bfvm_solver* m, int* num_densities);

/* Whole-field transfers of p_density_vectors (BioFVM_microenvironment.h:63),
 * host buffer [N][S] doubles.  In FP32 mode values are converted. */
BFVM_API int bfvm_set_densities(bfvm_solver* m, const double* host);
BFVM_API int bfvm_get_densities(bfvm_solver* m, double* host);
/* Per-voxel access, the device analogue of density_vector(n)
 * (BioFVM_microenvironment.cpp:499-500): values [count][S]. */
BFVM_API int bfvm_get_voxel_densities(bfvm_solver* m, int64_t count, const int64_t* voxels,
                             double* values);
BFVM_API int bfvm_set_voxel_densities(bfvm_solver* m, int64_t count, const int64_t* voxels,
                             const double* values);
/* The same gather as bfvm_get_voxel_densities, for callers that can't call
 * cudaMalloc (no counterpart in the reference, which has no device).
 * cudaMalloc and cudaFree can synchronise the whole device, which a host
 * loop that must not stall cannot afford, and where another allocator holds
 * the device's memory a fresh cudaMalloc may fail.  This entry point
 * allocates nothing: it stages the voxel list and the values in one 4 MiB
 * file-scope device array, so count*(8 + 8*S) bytes (the voxel list rounded
 * up to 256) must fit, else BFVM_ERR_ARG.  Every GPU that loads the library
 * holds that array until exit.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  All calls share the array and it keeps the last
 * call's contents; calls whose GPU work overlaps race on it (each call
 * synchronises the solver's stream before returning). */
BFVM_API int bfvm_get_voxel_densities_noalloc(bfvm_solver* m, int64_t count,
                                              const int64_t* voxels, double* values);
/* Device address of the density field ([N][S], double or float per the
 * precision); valid until the next resize or precision change. */
BFVM_API int bfvm_device_densities(bfvm_solver* m, void** device_ptr);

/* The three bulk callbacks bulk_supply_rate_function,
 * bulk_supply_target_densities_function, bulk_uptake_rate_function
 * (BioFVM_microenvironment.h:130-132), evaluated by the caller for every
 * voxel: [N][S] each, NULL = the reference default zero_function.  Voxels
 * whose supply and uptake are zero for every density are identities of
 * simulate_bulk_sources_and_sinks and are not stored. */
BFVM_API int bfvm_set_bulk_rates(bfvm_solver* m, const double* supply, const double* target,
                        const double* uptake);
/* Same, listing only the voxels with non-zero rates: [count][S] each. */
BFVM_API int bfvm_set_bulk_rates_sparse(bfvm_solver* m, int64_t count, const int64_t* voxels,
                               const double* supply, const double* target,
                               const double* uptake);

/* Microenvironment::add_dirichlet_node / update_dirichlet_node /
 * remove_dirichlet_node (BioFVM_microenvironment.cpp:146-189); value [S].
 * Nodes are applied in list order (a later node for the same voxel wins). */
BFVM_API int bfvm_add_dirichlet_node(bfvm_solver* m, int64_t voxel, const double* value);
BFVM_API int bfvm_update_dirichlet_node(bfvm_solver* m, int64_t voxel, const double* value);
BFVM_API int bfvm_remove_dirichlet_node(bfvm_solver* m, int64_t voxel);
BFVM_API int bfvm_clear_dirichlet_nodes(bfvm_solver* m);
BFVM_API int bfvm_get_num_dirichlet_nodes(bfvm_solver* m, int64_t* count);

/* The agents' cell_source_sink_solver_temp1/temp2 of
 * Basic_Agent::set_internal_uptake_constants (BioFVM_basic_agent.cpp:114-148)
 * with current_voxel_index, in agent-list order (all_basic_agents,
 * BioFVM_basic_agent.cpp:35): voxel[A], temp1[A][S], temp2[A][S]. */
BFVM_API int bfvm_set_agents(bfvm_solver* m, int64_t count, const int64_t* voxel, const double* temp1,
                    const double* temp2);
/* Densities at the agents' voxels, [A][S], agent order: the read a caller
 * makes through Basic_Agent::nearest_density_vector (BioFVM_basic_agent.cpp:223). */
BFVM_API int bfvm_get_agent_densities(bfvm_solver* m, double* values);

/* Asynchronous forms of the two calls above, for a host loop that exchanges
 * agent data with the solver every step (the reference's per-step
 * set_internal_uptake_constants and nearest_density_vector,
 * BioFVM_basic_agent.cpp:114-148, 223).  Both return at once.
 *
 * bfvm_set_agents_async: the copies of voxel/temp1/temp2 and the sort of the
 * agents by voxel run on the solver's upload stream, into a second device
 * buffer set, while steps enqueued earlier still run on the first; steps
 * enqueued after this call use the new agents.  The host arrays must stay
 * unchanged until bfvm_wait_transfers (or bfvm_synchronize) returns.
 *
 * bfvm_get_agent_densities_async: the densities at the agents' voxels as
 * they stand after the work enqueued so far, copied into values [A][S] on
 * the solver's download stream while later steps run; values holds them once
 * bfvm_wait_transfers (or bfvm_synchronize) returns.
 *
 * The copies overlap the steps when the host arrays are page-locked. */
BFVM_API int bfvm_set_agents_async(bfvm_solver* m, int64_t count, const int64_t* voxel,
                                   const double* temp1, const double* temp2);
BFVM_API int bfvm_get_agent_densities_async(bfvm_solver* m, double* values);
/* Waits for the transfers of the asynchronous calls enqueued so far. */
BFVM_API int bfvm_wait_transfers(bfvm_solver* m);

/* Microenvironment::simulate_bulk_sources_and_sinks
 * (BioFVM_microenvironment.cpp:584-613). */
BFVM_API int bfvm_simulate_bulk_sources_and_sinks(bfvm_solver* m, double dt);
/* Microenvironment::simulate_cell_sources_and_sinks
 * (BioFVM_microenvironment.cpp:615-633): agents applied in list order. */
BFVM_API int bfvm_simulate_cell_sources_and_sinks(bfvm_solver* m, double dt);
/* Microenvironment::simulate_diffusion_decay (BioFVM_microenvironment.cpp:502-513)
 * dispatching to diffusion_decay_solver__constant_coefficients_LOD_3D
 * (BioFVM_solvers.cpp:77-276). */
BFVM_API int bfvm_simulate_diffusion_decay(bfvm_solver* m, double dt);
/* diffusion_decay_solver__constant_coefficients_LOD_2D
 * (BioFVM_solvers.cpp:278-427): x and y sweeps of the z = 0 plane with the
 * decay split in halves; it shares the Thomas set-up with the 3-D solver as
 * the reference does. */
BFVM_API int bfvm_simulate_diffusion_decay_2d(bfvm_solver* m, double dt);
/* Microenvironment::apply_dirichlet_conditions (BioFVM_microenvironment.cpp:192-197). */
BFVM_API int bfvm_apply_dirichlet_conditions(bfvm_solver* m);
/* nsteps of the canonical step bulk -> cells -> diffusion
 * (examples/performance_test_numcells.cpp:177-179), fused into three sweep
 * kernels per step; flags selects the parts (BFVM_STEP_*). */
BFVM_API int bfvm_step(bfvm_solver* m, double dt, int nsteps, int flags);

/* ---- one field split by z planes over several solvers (no counterpart in
 * the reference, which holds a Microenvironment in one process) ----------
 *
 * The solver's mesh holds planes [bounds[rank], bounds[rank+1]) of a field
 * of bounds[nranks] planes (bounds[0] = 0; every slab at least one plane;
 * its mesh must have bounds[rank+1] - bounds[rank] planes along z).  x and y
 * lines lie in one plane and are solved by the slab alone; the z sweep of a
 * bfvm_step solves the slab's segment of every z line with the whole line's
 * Thomas rows and zero carries at the slab's ends.  After each step, every
 * slab's first and last plane are gathered from every solver (an all-gather
 * over NCCL by the caller) into a device array planes [nranks][2][nx*ny*S]
 * (first plane, then last, per slab, in rank order), and bfvm_zslab_fixup
 * joins the slabs: the result equals the unsplit solve to rounding.  A slab
 * steps one diffusion step per bfvm_step call.  nranks = 0 ends the split;
 * a resize ends it too.  FP64 fields; at most 64 slabs.  Call before the
 * first step (the Thomas set-up is redone). */
BFVM_API int bfvm_set_z_slab(bfvm_solver* m, int nranks, const int* bounds, int rank);
BFVM_API int bfvm_zslab_fixup(bfvm_solver* m, const double* planes);

/* The reference computes the Thomas coefficients on the first diffusion call
 * and never again (diffusion_solver_setup_done, BioFVM_solvers.cpp:87,172),
 * so later changes of dt, D or decay are ignored.  This keeps that behaviour
 * and offers the explicit reset the reference lacks. */
BFVM_API int bfvm_reset_diffusion_setup(bfvm_solver* m);

/* FP64 (default, the reference's arithmetic) or FP32 sweeps (coefficients
 * still computed in FP64, cell sources accumulated in FP64).  Converts the
 * resident field. */
BFVM_API int bfvm_set_precision(bfvm_solver* m, int precision);

/* Launch shape of one axis's sweep kernel (no counterpart in the reference,
 * whose OpenMP loops have no tunables): chunk = points per thread (8, 16,
 * 32), columns = lines per block (8..64), min_blocks = resident blocks per SM
 * the kernel is compiled for (1, 2).  Kept until the next resize.  The
 * default is chosen from the axis length; the autotuner sets this. */
BFVM_API int bfvm_set_sweep_config(bfvm_solver* m, int axis, int chunk, int columns,
                                   int min_blocks);
/* config[4] = chunk, columns, min_blocks, and the tiles in the x row
 * kernel's shared-memory ring (2, or 3 where the tuner found it faster) */
/* Tiles in the x row kernel's shared-memory ring: 2 (default) or 3 (one more
 * tile in flight while a tile is solved; fewer rows per tile where shared
 * memory runs short).  Kept until the next resize or tuning. */
BFVM_API int bfvm_set_row_stages(bfvm_solver* m, int stages);
/* Build of the x row kernel (a tuning choice with no counterpart in the
 * reference, like the ring depth above): 0 any density count; 1 a build for
 * exactly this density count, so that the offsets along a row are
 * compile-time constants; 2 (default) that build reading the chunk tables
 * in their planar layout.  Builds 1 and 2 exist for FP64 fields of 4, 8, 10
 * or 16 densities at 32-point chunks with the tables in shared memory, one
 * block per SM and a two-tile ring; elsewhere the row kernel runs build 0.
 * Same results bit for bit.  bfvm_tune_sweeps tries all three.  Kept until
 * the next resize or tuning. */
BFVM_API int bfvm_set_row_build(bfvm_solver* m, int build);
/* requested = the build set above; effective = the build the row kernel
 * runs under the current plan when it sweeps x (0 where builds 1 and 2 do
 * not apply, and before the first sweep has built the chunk tables). */
BFVM_API int bfvm_get_row_build(bfvm_solver* m, int* requested, int* effective);
/* Which sweep kernels run (all compute the same sweep):
 *   BFVM_PATH_AUTO    (default) the register kernel for x, the TMA-fed
 *                     persistent kernel for y and z where the layout allows
 *                     it (16-byte multiple row and plane strides), else
 *                     direct loads;
 *   BFVM_PATH_GENERIC the first, table-free register kernel on every axis;
 *   BFVM_PATH_TMA     TMA-fed persistent kernels on every axis they fit;
 *   BFVM_PATH_DIRECT  direct-load kernels on every axis. */
#define BFVM_PATH_AUTO 0
#define BFVM_PATH_GENERIC 1
#define BFVM_PATH_TMA 2
#define BFVM_PATH_DIRECT 3
BFVM_API int bfvm_set_kernel_path(bfvm_solver* m, int path);
/* bfvm_step: 0 (default) runs the bulk and cell updates as their own kernels
 * over the stored voxel lists before the x sweep; 1 applies them inside the
 * x sweep's prologue.  Same results either way. */
BFVM_API int bfvm_set_fuse_sources(bfvm_solver* m, int fuse);
BFVM_API int bfvm_get_fuse_sources(bfvm_solver* m, int* fuse);
BFVM_API int bfvm_get_sweep_config(bfvm_solver* m, int axis, int* config);

BFVM_API int bfvm_synchronize(bfvm_solver* m);
/* The solver's cudaStream_t, for events and interop. */
BFVM_API int bfvm_get_stream(bfvm_solver* m, void** stream);
/* Kernel launches enqueued by this solver since creation. */
BFVM_API int bfvm_get_launch_count(bfvm_solver* m, int64_t* count);

/* Sweep tuner (no counterpart in the reference): for each axis, times every
 * kernel that can run it -- the register kernel at each chunk length and
 * block width, the TMA-fed kernel and the direct kernel at each chunk
 * length -- over reps sweeps of this solver's own field, and keeps the
 * fastest for later steps (used while the kernel path is BFVM_PATH_AUTO);
 * then the slab thickness of bfvm_set_slab_planes and bfvm_set_fuse_sources,
 * over whole steps.
 * The field is saved before and restored after; bfvm_set_sweep_config or
 * a resize resets the choice.  bfvm_get_sweep_kernel returns the axis's
 * kernel (0 = the default choice, else a BFVM_PATH_* value). */
BFVM_API int bfvm_tune_sweeps(bfvm_solver* m, double dt, int reps);
BFVM_API int bfvm_get_sweep_kernel(bfvm_solver* m, int axis, int* kind);

/* Runs the x and y sweeps of a step slab by slab: for each slab of `planes`
 * z planes the x sweep, then the y sweep (an x line and a y line lie in one
 * plane, so the y sweep of a slab needs only that slab's x sweep).  A slab
 * that fits in L2 is written by the x sweep and read back by the y sweep
 * from L2, so the field crosses HBM once for both sweeps instead of twice.
 * 0 (the default) sweeps whole axes; bfvm_tune_sweeps also picks this.
 * Results equal the whole-axis sweeps' to the last bit whenever the same
 * kernels run. */
BFVM_API int bfvm_set_slab_planes(bfvm_solver* m, int planes);
BFVM_API int bfvm_get_slab_planes(bfvm_solver* m, int* planes);

/* Self-test of the TMA sweeps' error path on `device`: a kernel waits on a
 * barrier that nothing completes, with the sweeps' bounded wait limited to
 * limit_ns (1 us .. 2 s); the wait gives up and the kernel returns with its
 * status set, as a sweep that gave up waiting for a copy would.
 * *gave_up = 1 when the status came back set, *waited_ms = the kernel's
 * time.  The device stays usable afterwards. */
BFVM_API int bfvm_selftest_bounded_wait(int device, int64_t limit_ns, int* gave_up,
                                        double* waited_ms);

/* Whole steps of a small field in one thread-block cluster: under
 * BFVM_PATH_AUTO, bfvm_step runs all its steps in one launch when the FP64
 * field fits in the shared memory of a cluster of at most 8 blocks (about
 * 1.6 MB) and no axis has more than 64 points.  The field stays in shared
 * memory across the steps; z lines are solved through distributed shared
 * memory; lines use the reference's own operation sequence (bit-exact).
 * enable = 1 turns it on (off by default: it is a bit-exact mode, slower
 * than the sweep kernels -- 103 vs 25 us per step at 50^3 on a B200);
 * bfvm_get_cluster_steps gives the cluster's block count for this solver
 * now (0: not used). */
BFVM_API int bfvm_set_cluster_steps(bfvm_solver* m, int enable);
BFVM_API int bfvm_get_cluster_steps(bfvm_solver* m, int* blocks);

/* Whole steps of a small field in one cooperative launch over all SMs: under
 * BFVM_PATH_AUTO, bfvm_step runs all its steps in one launch when the FP64
 * field has at most 2^19 voxel-densities and no axis has more than 64
 * points (and the cluster mode above is not in use).  Each step is a phase of
 * bulk and cell updates, then one phase per axis in which blocks solve tiles
 * of lines in 4- or 8-point chunks as the sweep kernels do (Dirichlet values applied
 * as the chunks load), separated by grid-wide barriers; after the first
 * step the bulk and cell updates are applied as the previous z phase stores
 * its points.  On by default (17.7 vs 24.7 us per step at 50^3 x 1 on a
 * B200 with 1000 agents, faster than the sweep
 * kernels up to 2^19 voxel-densities); enable = 0 gives back the sweep
 * kernels.  bfvm_get_grid_steps gives the launch's block count for this
 * solver now (0: not used). */
BFVM_API int bfvm_set_grid_steps(bfvm_solver* m, int enable);
BFVM_API int bfvm_get_grid_steps(bfvm_solver* m, int* blocks);

/* Times bfvm_step's kernels with CUDA events on the solver's stream, averaged
 * over nsteps steps: ms[4] = source kernels (bulk + cells), x sweep (with its
 * Dirichlet prologue/epilogue), y sweep, z sweep.  With slabs
 * (bfvm_set_slab_planes) the x entry holds the x and y sweeps together and
 * the y entry is 0. */
BFVM_API int bfvm_profile_step(bfvm_solver* m, double dt, int nsteps, int flags, double* ms);

/* Microenvironment::compute_all_gradient_vectors (BioFVM_microenvironment.cpp:
 * 702-787): central differences (p[n+jump] - p[n-jump]) / (2 dx) along each
 * axis at the points with a neighbour on both sides, into the solver's
 * device gradient array [N][S][3] (FP64).  Components of points at an axis
 * end keep their previous values (zero when the array is first made; the
 * array is kept across steps, widened by add_density, cleared by resize).
 * The reference takes its jumps from the LOD_3D setup and its 2 dx from the
 * first mesh it sees (static constants); here they are the current mesh's. */
BFVM_API int bfvm_compute_all_gradient_vectors(bfvm_solver* m);
BFVM_API int bfvm_get_gradient_vectors(bfvm_solver* m, double* out);
BFVM_API int bfvm_device_gradients(bfvm_solver* m, void** ptr);

/* ---- derivatives (no counterpart in the reference) ----------------------
 *
 * bfvm_adjoint_forward runs nsteps steps exactly like bfvm_step(m, dt,
 * nsteps, flags) (FP64 only) and keeps the field every checkpoint_every
 * steps.  bfvm_adjoint_backward then takes seed = dLoss/d(final field)
 * ([N][S] FP64; host memory, or device memory when seed_on_device != 0) and
 * returns, in host arrays (each may be NULL):
 *   grad_D[S], grad_decay[S]       dLoss/d(diffusion coefficient, decay rate)
 *   grad_temp1[A*S], grad_temp2[A*S]  dLoss/d(agent temp1, temp2), agents in
 *       list order (Basic_Agent::cell_source_sink_solver_temp1/2,
 *       BioFVM_basic_agent.cpp:139-147)
 *   grad_p0[N*S]                   dLoss/d(field before the first step)
 * It recomputes each checkpoint segment (3 fields kept per step of a
 * segment) and applies the adjoint step by step in reverse.  The solver must
 * not change between the two calls; the field keeps the forward result. */
BFVM_API int bfvm_adjoint_forward(bfvm_solver* m, double dt, int nsteps, int flags,
                                  int checkpoint_every);
BFVM_API int bfvm_adjoint_backward(bfvm_solver* m, const double* seed, int seed_on_device,
                                   double* grad_D, double* grad_decay, double* grad_temp1,
                                   double* grad_temp2, double* grad_p0);
/* Frees the checkpoints and buffers of the adjoint. */
BFVM_API int bfvm_adjoint_release(bfvm_solver* m);

/* ---- many independent microenvironments (no counterpart in the reference,
 * whose drivers loop over Microenvironment objects one by one) ----------
 *
 * A batch refers to solvers (not owned; they must outlive their batch
 * membership) of one device and one precision.  bfvm_batch_step(b, dt, n,
 * flags) has the effect of bfvm_step(m, dt, n, flags) on every member: the
 * instances are packed into groups whose fields fit a byte budget (default
 * half the L2 cache) and every phase of a step is one launch over a group;
 * the groups x steps x phases sequence is captured into a CUDA graph and
 * replayed by one graph launch (the graph is kept while the plan is
 * unchanged).  Work already queued on a member's stream runs first; later
 * calls on a member wait for the batch. */
typedef struct bfvm_batch bfvm_batch;
BFVM_API int bfvm_batch_create(bfvm_batch** out, int device);
BFVM_API int bfvm_batch_destroy(bfvm_batch* b);
BFVM_API int bfvm_batch_add(bfvm_batch* b, bfvm_solver* m);
BFVM_API int bfvm_batch_clear(bfvm_batch* b);
BFVM_API int bfvm_batch_size(bfvm_batch* b, int* count);
BFVM_API int bfvm_batch_step(bfvm_batch* b, double dt, int nsteps, int flags);
/* Autotuner: times short graph runs (trial_steps steps) of candidate chunk
 * lengths x threads per block for each axis, tunes every member's own sweeps
 * (bfvm_tune_sweeps, which branch mode runs), then candidate group budgets
 * in every mode (BFVM_BATCH_FUSED, BFVM_BATCH_BRANCHES, BFVM_BATCH_PERSISTENT
 * at each chunk length, BFVM_BATCH_PLANES), and keeps the fastest.  The members' fields are saved before and restored
 * after, so tuning does not advance the simulation. */
BFVM_API int bfvm_batch_tune(bfvm_batch* b, double dt, int flags, int trial_steps);
/* chunk[3] in {8,16,32} with threads[3] in {128,256,512} per axis, or 0/0 to
 * choose; group_bytes -1 = default, 0 = all members in one group. */
BFVM_API int bfvm_batch_set_config(bfvm_batch* b, const int* chunk, const int* threads,
                                   int64_t group_bytes);
BFVM_API int bfvm_batch_get_config(bfvm_batch* b, int* chunk, int* threads, int64_t* group_bytes);
/* How a group of members runs (the whole call stays one CUDA-graph launch):
 *   BFVM_BATCH_FUSED       every phase of a step is one launch over all of
 *                          the group's members (default);
 *   BFVM_BATCH_BRANCHES    every member runs its own single-instance kernels
 *                          (its own sweep choices, bfvm_tune_sweeps) on its
 *                          own branch of the graph; the branches of a group
 *                          run concurrently;
 *   BFVM_BATCH_PERSISTENT  all n steps of every member of a group in ONE
 *                          persistent cooperative launch over all SMs: the
 *                          phases of a step (first-step sources, x, y, z
 *                          with the next step's sources on the z stores)
 *                          are shared by the members and separated by grid
 *                          barriers, so a group that fits L2 keeps its fields
 *                          on chip for the whole call.  Members with an FP64
 *                          field and lines of at most 128 points; the others
 *                          run as in BFVM_BATCH_BRANCHES, after the
 *                          persistent groups.
 *   BFVM_BATCH_PLANES      as BFVM_BATCH_PERSISTENT (one cooperative launch
 *                          per group for all n steps), with two phases per
 *                          step: xy planes of a member (all its densities,
 *                          or as many as fit 111 KB of shared memory) are
 *                          staged in shared memory and solved along x, then
 *                          y, one thread per whole line; then strips of xz
 *                          planes are staged and solved along z, the next
 *                          step's sources applied as the points are
 *                          stored.  The field crosses L2 twice per step.
 *                          Members with an FP64 field, lines of at most 128
 *                          points and planes that fit; the others run as in
 *                          BFVM_BATCH_BRANCHES.
 * bfvm_batch_tune chooses between them. */
#define BFVM_BATCH_FUSED 0
#define BFVM_BATCH_BRANCHES 1
#define BFVM_BATCH_PERSISTENT 2
#define BFVM_BATCH_PLANES 3
BFVM_API int bfvm_batch_set_mode(bfvm_batch* b, int mode);
BFVM_API int bfvm_batch_get_mode(bfvm_batch* b, int* mode);
/* Work split of the persistent mode's kernel: chunks of 8 (default) or 16
 * points per thread, folded across the threads of a block; 32, tiles of 32
 * columns x at most 4 chunks of 32 points solved with the sweep kernels'
 * chunk tables; or 0, one thread per (line, density) column solving the
 * whole line (no fold, the field read and written twice per sweep).
 * bfvm_batch_tune also picks it. */
BFVM_API int bfvm_batch_set_persistent_chunk(bfvm_batch* b, int chunk);
BFVM_API int bfvm_batch_get_persistent_chunk(bfvm_batch* b, int* chunk);
/* Groups of the last plan and kernel launches in its graph. */
BFVM_API int bfvm_batch_get_plan(bfvm_batch* b, int* groups, int64_t* kernels_per_call);
BFVM_API int bfvm_batch_synchronize(bfvm_batch* b);

#ifdef __cplusplus
}
#endif
#endif
