/*
 * icempm_b200 — C-ABI of the B200-native single-partition MLS-MPM step.
 *
 * Plain C: an opaque handle, plain pointers and sizes, int status returns.
 * No exception crosses this boundary. One host thread drives a handle; all
 * device work of a handle is issued on one CUDA stream (its own, or the one
 * given to mpm_set_stream).
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the reference project root).
 *
 * Status codes
 *   0          ok
 *   70..75     a particle left the grid in -x/-y/-z/+x/+y/+z
 *              (the device error byte of mpm_kernels.cuh:70-75)
 *   5          receive overflow (mpm_kernels.cuh:420; never raised with one
 *              partition, kept for the numbering)
 *   >= 100     new codes of this library, listed below
 */
#ifndef ICEMPM_B200_H
#define ICEMPM_B200_H

#include <stddef.h>
#include <stdint.h>
#include "sim_params_3d.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_OK                 0
#define MPM_ERR_RECEIVE        5
#define MPM_ERR_OUT_XMIN      70
#define MPM_ERR_OUT_YMIN      71
#define MPM_ERR_OUT_ZMIN      72
#define MPM_ERR_OUT_XMAX      73
#define MPM_ERR_OUT_YMAX      74
#define MPM_ERR_OUT_ZMAX      75
#define MPM_ERR_CUDA         100  /* a CUDA runtime call failed              */
#define MPM_ERR_ARG          101  /* invalid argument (null, size, mode)     */
#define MPM_ERR_CAPACITY     102  /* more particles than the handle holds    */
#define MPM_ERR_NO_DEVICE    103  /* no CUDA device / wrong architecture     */
#define MPM_ERR_CONFIG_FILE  104  /* configuration file missing / unreadable */
#define MPM_ERR_CONFIG_JSON  105  /* not JSON, or a key of the wrong type    */
#define MPM_ERR_CONFIG_KEY   106  /* required key "InputRawPoints" missing   */
#define MPM_ERR_SORT_RANGE   107  /* a particle's cell key lies outside grid */
#define MPM_ERR_STATE        108  /* call out of order (e.g. step before upload) */
#define MPM_ERR_NOALLOC_LIMIT 109 /* size beyond the fixed scratch of mpm_sort_permutation_noalloc */

#define MPM_PRECISION_FP64   0    /* FP64 state and transfers; 3x3 SVD in FP32
                                     exactly as the reference (helper_math.cuh) */
#define MPM_PRECISION_MIXED  1    /* FP32 state and transfers; the grid is
                                     accumulated with plain FP32 float4
                                     atomics (same-cell particle pairs merged
                                     in registers first): no compensated or
                                     fixed-point sum; FP64 SVD, apex return
                                     map and indenter force reduction        */
#define MPM_PRECISION_FP64_SVD64 2 /* FP64 throughout, SVD included: the
                                     high-accuracy reference of the mixed mode */

typedef struct mpm_handle mpm_handle;

/* ---------------------------------------------------------------- params */

/* SimParams3D::Reset (parameters_sim_3d.cpp:5-62). */
void mpm_params_reset(SimParams3D* prms);
/* SimParams3D::ComputeLame (parameters_sim_3d.cpp:164-169). */
void mpm_params_compute_lame(SimParams3D* prms);
/* SimParams3D::ComputeCamClayParams (parameters_sim_3d.cpp:171-175). */
void mpm_params_compute_camclay(SimParams3D* prms);
/* SimParams3D::ComputeHelperVariables (parameters_sim_3d.cpp:65-86). */
void mpm_params_compute_helper_variables(SimParams3D* prms);
/* SimParams3D::SetPhi (parameters_sim_3d.h:100), angle in degrees. */
void mpm_params_set_phi(SimParams3D* prms, double phi_degrees);
/* SimParams3D::ParseFile (parameters_sim_3d.cpp:89-162): Reset, then read the
 * same JSON keys, then derive. The value of "InputRawPoints" is copied into
 * raw_points_file (NUL-terminated, truncated to buflen). Returns 0, or
 * MPM_ERR_CONFIG_FILE / _JSON / _KEY where the reference throws. */
int  mpm_params_parse_file(SimParams3D* prms, const char* path,
                           char* raw_points_file, int buflen);
/* Same as mpm_params_parse_file on an in-memory JSON text. */
int  mpm_params_parse_string(SimParams3D* prms, const char* json_text,
                             char* raw_points_file, int buflen);

/* ---------------------------------------------------------------- handle */

/* GPU_Implementation6::initialize (gpu_implementation6.cpp:319-337),
 * GPU_Implementation6::allocate_arrays (:385-401),
 * GPU_Implementation6::update_constants (:522-525) and
 * GPU_Partition_3D::initialize (gpu_partition_3d.cu:52-73),
 * GPU_Partition_3D::allocate (:76-132), GPU_Partition_3D::update_constants
 * (:135-143). One partition on `device`.
 * `capacity` = number of particles the handle can hold. The grid is the
 * reference's one-partition buffer, (GridXTotal + 2 GridHaloSize) x GridY x
 * GridZ nodes (GridHaloSize = 0 needs no halo slabs with one partition),
 * fewer than 2^31 of them. MPM_PRECISION_MIXED holds positions as x / h in
 * 32-bit fixed point with 20 fraction bits: each grid dimension (x with its
 * halo slabs) must be below 2047 cells. Otherwise MPM_ERR_ARG.
 * *status receives 0 or an error code; NULL is returned on error. */
mpm_handle* mpm_create(const SimParams3D* prms, int precision, unsigned capacity,
                       int device, int* status);
/* GPU_Partition_3D::~GPU_Partition_3D (gpu_partition_3d.cu:27-50). */
void mpm_destroy(mpm_handle* h);
/* Issue all later work of h on `cuda_stream` (a cudaStream_t); NULL restores
 * the handle's own stream. */
int  mpm_set_stream(mpm_handle* h, void* cuda_stream);
/* GPU_Implementation6::update_constants (gpu_implementation6.cpp:522-525),
 * GPU_Partition_3D::update_constants (gpu_partition_3d.cu:135-143): copies
 * the parameter block to the device and clears the device error byte. The
 * grid dimensions must not change. */
int  mpm_update_constants(mpm_handle* h, const SimParams3D* prms);

/* -------------------------------------------------------- particle data */

/* HostSideSOA::Allocate (host_side_soa.cpp:70-86) allocates the host SoA as
 * page-locked memory (cudaMallocHost), so that the uploads and downloads of
 * the SoA run at the host link's speed. mpm_host_alloc gives such memory to
 * a host that does not link CUDA itself: *ptr receives bytes of page-locked
 * host memory (NULL for bytes == 0). Release it with mpm_host_free, as the
 * reference does with cudaFreeHost (host_side_soa.cpp:72). */
int  mpm_host_alloc(size_t bytes, void** ptr);
int  mpm_host_free(void* ptr);

/* GPU_Implementation6::transfer_ponts_to_device (gpu_implementation6.cpp:404-414),
 * GPU_Partition_3D::transfer_points_from_soa_to_device (gpu_partition_3d.cu:201-215):
 * n particles from a host SoA in the reference's HostSideSOA row layout
 * (row k at soa + k*pitch, 28 rows). */
int  mpm_upload_soa(mpm_handle* h, const double* soa, unsigned pitch, unsigned n);
/* New per-particle field (no reference counterpart): cohesion c_i in Pa.
 * The Drucker-Prager apex shift becomes p0_i = c_i / DP_tan_phi in place of
 * the global DP_threshold_p (mpm_kernels.cuh:499,505-509,525). NULL clears
 * the field and restores the global value. */
int  mpm_upload_cohesion(mpm_handle* h, const double* cohesion, unsigned n);
/* GPU_Implementation6::transfer_from_device (gpu_implementation6.cpp:417-496),
 * GPU_Partition_3D::transfer_from_device (gpu_partition_3d.cu:169-199):
 * writes the particles in the handle's current order into the host SoA
 * (28 rows, row stride pitch >= n), *n = count.
 * Returns the device error code (70..75) if one was raised, as the
 * reference throws on it. */
int  mpm_download_soa(mpm_handle* h, double* soa, unsigned pitch, unsigned* n);
/* New: the upload index of each particle in the current order (the sort of
 * mpm_sort permutes particles; this gives the permutation). */
int  mpm_download_ids(mpm_handle* h, unsigned* ids, unsigned* n);
/* New: replaces the ids of the n particles the handle holds (n must be its
 * count), e.g. with global indices of a partitioned run. */
int  mpm_upload_ids(mpm_handle* h, const unsigned* ids, unsigned n);
/* New: the per-particle cohesion c_i (p0_i * DP_tan_phi) in the handle's
 * current order; MPM_ERR_STATE when none was uploaded. */
int  mpm_download_cohesion(mpm_handle* h, double* cohesion, unsigned* n);
/* HostSideSOA::RemoveDisabledAndSort (host_side_soa.cpp:56-67) on the device:
 * drops disabled particles and orders the rest by the cell key of
 * ProxyPoint3D::getCellIndex (proxypoint3d.cpp:158-163), stable (ties keep
 * their previous order). */
int  mpm_sort(mpm_handle* h);
/* New (no reference counterpart): the grid accumulator of the mixed P2G.
 * MPM_ACCUM_FLOAT (default): float4 {m, m v} per node, FP32 vector atomics,
 * whose rounding depends on the order of the adds. MPM_ACCUM_FIXED: each
 * contribution in 64-bit fixed point (2^44 units per the larger particle
 * mass, and per that mass at vmax for momentum), added as integers: the sums
 * are exact and independent of the order, and a run repeats bit for bit in
 * its particle state; 32 B per node instead of 16. FP64 handles accept only
 * MPM_ACCUM_FLOAT (their FP64 sums are kept as they are). */
#define MPM_ACCUM_FLOAT 0
#define MPM_ACCUM_FIXED 1
int  mpm_set_grid_accumulation(mpm_handle* h, int mode);
/* Sort automatically every k substeps inside mpm_step (0 = never, the
 * default, as with one partition the reference never re-sorts). */
int  mpm_set_sort_interval(mpm_handle* h, int k);

/* ------------------------------------------------ animation-frame records */

/* The records of SnapshotManager::SaveFrame (snapshotmanager.cpp:116-293) in
 * the reference's memory layout (converter/visualpoint.h:7-11,
 * snapshotmanager.h:30-36): VisualPoint, std::pair<int, std::array<float,6>>,
 * std::pair<int, float>, std::pair<int, uint8_t>. */
typedef struct { float pos[3], vel[3], Jp_inv; uint8_t status, pad[3]; } mpm_visual_point;   /* 32 bytes */
typedef struct { int32_t idx; float pos[3], vel[3]; } mpm_update_pos;                          /* 28 bytes */
typedef struct { int32_t idx; float Jp_inv; } mpm_update_jp;                                   /*  8 bytes */
typedef struct { int32_t idx; uint8_t status, pad[3]; } mpm_update_status;                     /*  8 bytes */

/* SaveFrame's change detection, on the device. The visual index of a
 * particle is its rank among the non-disabled particles in the handle's
 * current order; status byte = partition id (bits 24-31 of the status word)
 * | 0x80 if crushed; positions, velocities and Jp_inv are cast to float.
 * full != 0 (SaveFrame without a previous frame): keeps every particle as
 * the visual state, with `frame` as its last position refresh, and copies
 * the VisualPoint records to `points` (*n_points of them; room for the
 * particle count). full == 0 (needs a full frame since the last
 * mpm_upload_soa, else MPM_ERR_STATE): for each particle, in order,
 *   |pos - (vpos + vvel * (float)(dt * (frame - last) * UpdateEveryNthStep))|
 *   > animation_threshold_pos -> an UpdatePos record, last = frame;
 *   |vJp_inv - Jp_inv| > 1e-2  -> an UpdateJp record;
 *   status byte changed        -> an UpdateStatus record;
 * each output holds room for the particle count, the counts are returned.
 * As in the reference (which updates a copy of visual_state[count]), a
 * partial frame changes only `last`; the kept positions, velocities,
 * Jp_inv and status bytes stay those of the last full frame. */
int  mpm_frame_records(mpm_handle* h, int frame, int full, mpm_visual_point* points, unsigned* n_points,
                       mpm_update_pos* upd_pos, unsigned* n_pos, mpm_update_jp* upd_jp, unsigned* n_jp,
                       mpm_update_status* upd_status, unsigned* n_status);

/* ------------------------------------------ substep phases (one partition) */

/* GPU_Implementation6::reset_grid (gpu_implementation6.cpp:18-29). */
int  mpm_reset_grid(mpm_handle* h);
/* GPU_Implementation6::p2g (gpu_implementation6.cpp:31-77). */
int  mpm_p2g(mpm_handle* h);
/* GPU_Implementation6::update_nodes (gpu_implementation6.cpp:115-123); the
 * indenter centre is passed by value as GPU_Partition_3D::update_nodes
 * (gpu_partition_3d.cu:243-255) passes it. */
int  mpm_update_nodes(mpm_handle* h, double indenter_x, double indenter_y);
/* GPU_Implementation6::g2p (gpu_implementation6.cpp:125-133); record_pq as
 * recordPQ (mpm_kernels.cuh:347-351). */
int  mpm_g2p(mpm_handle* h, int record_pq);
/* GPU_Implementation6::reset_indenter_force_accumulator (gpu_implementation6.cpp:527-534),
 * GPU_Partition_3D::reset_indenter_force_accumulator (gpu_partition_3d.cu:145-150). */
int  mpm_reset_indenter_force_accumulator(mpm_handle* h);

/* ---------------------------------------------------------------- driver */

/* The substep loop of Model3D::Step (model_3d.cpp:24-112, the loop at :35-51) for nsteps
 * substeps: SimulationTime += dt; indenter_x = indenter_x_initial +
 * SimulationTime*IndVelocity; reset grid, P2G, grid update, G2P (P,Q
 * recorded when SimulationStep % UpdateEveryNthStep == 0);
 * SimulationStep += 1. force_hist (host, may be NULL) receives nsteps x 3
 * doubles: the total force on the indenter of each substep (sum over the
 * sensor bins of that substep, N). Returns the device error code if one was
 * raised during these substeps. */
int  mpm_step(mpm_handle* h, int nsteps, double* force_hist);
/* The frame-level sensor readout of GPU_Implementation6::transfer_from_device
 * (gpu_implementation6.cpp:417-496, the sensor at :438-459): sensor receives
 * 3*IndenterSubdivisions*GridZ doubles, each divided by
 * UpdateEveryNthStep*cellsize^2; total receives the summed force divided by
 * UpdateEveryNthStep (GPU_Implementation6::evaluate_indenter_total_force,
 * gpu_implementation6.cpp:499-510). */
int  mpm_sensors(mpm_handle* h, double* sensor, double total[3]);
/* The device error byte (gpu_error_indicator, mpm_kernels.cuh:17). */
int  mpm_get_error(mpm_handle* h);
/* GPU_Implementation6::synchronize (gpu_implementation6.cpp:513-520). */
int  mpm_synchronize(mpm_handle* h);
/* Read back the handle's copy of the parameter block (SimulationTime,
 * SimulationStep, indenter_x advance inside mpm_step). */
int  mpm_get_params(mpm_handle* h, SimParams3D* out);
/* Number of particles currently held (after sorts that drop disabled ones). */
int  mpm_count(mpm_handle* h, unsigned* n);
/* ------------------------------------------------ x-slab partitions
 * nPartitions > 1: the particles are split into slabs of grid columns along
 * x; after P2G neighbouring partitions add each other's 2*GridHaloSize
 * boundary slabs, and particles that leave a slab move to the neighbour.
 * Each partition keeps a grid of the whole domain and works on its window
 * of it (the same node indices in every partition). GridHaloSize >= 3. */

/* GPU_Partition_3D's slab (GPU_Implementation6::split_hssoa_into_partitions,
 * gpu_implementation6.cpp:340-382): partition `id` (0..255) owns the grid
 * columns [x0, x0 + gxp) of GridXTotal and works on them with GridHaloSize
 * halo columns on each side. Particles are checked against base x in
 * [x0 - halo, x0 + gxp + halo - 3] (70 / 73 outside), the node update covers
 * the window's columns, and the indenter force of a node is counted by the
 * partition that owns its column only (the first and the last partition
 * also own the halo columns beyond the grid's ends); the reference, whose
 * partitions update their overlap alike, adds the overlap nodes' force of
 * both partitions (gpu_implementation6.cpp:450-455). id_base: the upload
 * index the next mpm_upload_soa gives its first particle (ids are global
 * across partitions). x0 = 0, gxp = GridXTotal is the one-partition default. */
int  mpm_set_partition(mpm_handle* h, int id, int x0, int gxp, unsigned id_base);
/* Bytes of one side's halo: 2*GridHaloSize*GridY*GridZ nodes, 32 B each
 * (FP64: 4 arrays) or 16 B (mixed: the float4 accumulator). */
size_t mpm_halo_bytes(const mpm_handle* h);
/* The halo sends of GPU_Implementation6::p2g (gpu_implementation6.cpp:31-77):
 * copies the P2G sums of the 2*GridHaloSize columns around the window's left
 * (side 0: x0 - halo .. x0 + halo - 1) or right (side 1: x0 + gxp - halo ..
 * x0 + gxp + halo - 1) boundary into the device buffer dst (mpm_halo_bytes;
 * FP64: the 4 arrays one after another). */
int  mpm_halo_pack(mpm_handle* h, int side, void* dst);
/* partition_kernel_receive_halos_left (mpm_kernels.cuh:103-118) and
 * partition_kernel_receive_halos_right (:120-135): adds a neighbour's packed
 * slabs of the same columns (its side 1 for our side 0 and vice versa) into
 * this grid. Addition commutes, so both partitions then hold equal sums. */
int  mpm_halo_add(mpm_handle* h, int side, const void* src);
/* Bytes of one particle record of a point transfer: 256 (FP64: the 28 SoA
 * rows, the apex shift p0, the id) or 128 (mixed: the 28 rows of the mixed
 * state, p0, the id). */
size_t mpm_point_record_bytes(const mpm_handle* h);
/* The point transfer of partition_kernel_g2p (mpm_kernels.cuh:353-398) and
 * PreparePointForTransfer (:401-408), run after a G2P: a particle whose base x
 * lies more than 3 columns left of x0, or right of x0 + gxp, is copied as a
 * record into left / right (device buffers of `capacity` records each) and
 * disabled (its status word set to the disabled bit). Only sides with a
 * neighbour (x0 > 0; x0 + gxp < GridXTotal) send. *n_left, *n_right: the
 * records written (at most capacity: a particle beyond a full buffer stays,
 * as in the reference); *max_deviation (may be NULL): the largest distance in
 * columns of a particle beyond the slab by more than halo/2 - 1 columns
 * (the reference's idx_pts_max_extent). Waits for the device. */
int  mpm_points_out(mpm_handle* h, void* left, void* right, unsigned capacity, unsigned* n_left, unsigned* n_right,
                    int* max_deviation);
/* partition_kernel_receive_points (mpm_kernels.cuh:411-427): appends `count`
 * records (device buffer) after the handle's particles; MPM_ERR_RECEIVE (5)
 * if they do not fit in its capacity. */
int  mpm_points_in(mpm_handle* h, const void* records, unsigned count);

/* The two halves of a substep of one partition, for a driver that runs the
 * halo exchange between them itself (one partition per process).
 * mpm_substep_p2g: the P2G sums of the current state in the grid (the first
 * half of GPU_Implementation6::p2g, gpu_implementation6.cpp:31-77; FP64:
 * window cleared, P2G; mixed: computed by the previous substep's fused
 * kernel, else a standalone P2G). */
int  mpm_substep_p2g(mpm_handle* h);
/* The rest of the substep of Model3D::Step (model_3d.cpp:24-112, the loop at
 * :35-51): SimulationTime += dt, the indenter moves, node update, G2P (mixed:
 * fused with the next substep's P2G), SimulationStep += 1. store_vc (mixed):
 * write v and C to the state (needed before a download or a point transfer).
 * force3 (host, may be NULL: no wait) receives the substep's force of the
 * nodes this partition owns. */
int  mpm_substep_update_g2p(mpm_handle* h, int store_vc, double force3[3]);

/* GPU_Implementation6 with prms->nPartitions partitions in one process:
 * GPU_Implementation6::initialize (gpu_implementation6.cpp:319-337) puts
 * partition i on devices[i % ndevices]; GPU_Implementation6::allocate_arrays
 * (:385-401) with `capacity` particles per partition (nPtsTotal /
 * nPartitions * (1 + ExtraSpaceForIncomingPoints) in the reference) and
 * VectorCapacity_transfer records per direction;
 * GPU_Implementation6::enable_peer_access (:219-315) for neighbours on other
 * devices. */
typedef struct mpm_multi mpm_multi;
mpm_multi* mpm_multi_create(const SimParams3D* prms, int precision, unsigned capacity, const int* devices,
                            int ndevices, int* status);
void mpm_multi_destroy(mpm_multi* m);
/* HostSideSOA::RemoveDisabledAndSort (host_side_soa.cpp:56-67), as a
 * stable sort here, then GPU_Implementation6::split_hssoa_into_partitions
 * (gpu_implementation6.cpp:340-382) and
 * GPU_Implementation6::transfer_ponts_to_device (gpu_implementation6.cpp:404-414)
 * of a host SoA in the HostSideSOA row layout: partition i takes
 * [n - done] / [N - i] particles, its slab ends at the x index of the next
 * partition's first particle, and bits 24-31 of the status word get i.
 * cohesion (may be NULL) as mpm_upload_cohesion. The upload index of each
 * particle is its id. */
int  mpm_multi_upload_soa(mpm_multi* m, const double* soa, unsigned pitch, unsigned n, const double* cohesion);
/* Model3D::Step (model_3d.cpp:24-112) for nsteps substeps: per substep P2G,
 * the halo exchange (GPU_Implementation6::p2g, gpu_implementation6.cpp:31-77;
 * GPU_Implementation6::receive_halos, :80-112), the node update, G2P, and
 * every UpdateEveryNthStep / PointTransferFrequency substeps the point
 * transfer (GPU_Implementation6::receive_points, :135-208); at the end of
 * each animation frame PointTransferFrequency grows when a particle strayed
 * more than GridHaloSize/2 columns, and the partitions are rebalanced
 * (RemoveDisabledAndSort, split, upload; model_3d.cpp:76-108) when one has
 * less than RebalanceThresholdFreeSpaceRemaining of free room or more than
 * RebalanceThresholdDisabledPercentage of its capacity disabled.
 * force_hist: nsteps x 3 forces summed over the partitions. */
int  mpm_multi_step(mpm_multi* m, int nsteps, double* force_hist);
/* GPU_Implementation6::transfer_from_device (gpu_implementation6.cpp:417-496):
 * the partitions' particles one after another (disabled ones included), row
 * stride pitch, and (ids may be NULL) the upload index of each; *n = count.
 * soa = NULL only returns the count. */
int  mpm_multi_download_soa(mpm_multi* m, double* soa, unsigned pitch, unsigned* ids, unsigned* n);
/* The rebalance of Model3D::Step (model_3d.cpp:24-112, the rebalance at
 * :99-108) on request. */
int  mpm_multi_rebalance(mpm_multi* m);
/* Partition i's slab [x0, x0 + gxp), its particle count (disabled included)
 * and its disabled count since the last split (nPts_disabled). */
int  mpm_multi_info(mpm_multi* m, int i, int* x0, int* gxp, unsigned* n, unsigned* n_disabled);
/* The largest transfer of one partition to one side, the rebalances so far
 * and the current PointTransferFrequency. */
int  mpm_multi_stats(mpm_multi* m, int* max_sent, int* rebalances, int* point_transfer_frequency);
/* mpm_sensors summed over the partitions. */
int  mpm_multi_sensors(mpm_multi* m, double* sensor, double total[3]);
/* mpm_reset_indenter_force_accumulator on every partition. */
int  mpm_multi_reset_indenter_force_accumulator(mpm_multi* m);

/* ---------------------------------------------------------------- adjoint
 * No counterpart in the reference (new, for calibrating ice strength).
 * Reverse-mode gradients of a loss on the indenter force history with
 * respect to per-particle cohesion and Young's modulus, through the FP64 step
 * (FP64 SVD). On a mixed handle the forward runs in mixed precision and the
 * reverse sweep recomputes each segment in FP64 from its checkpoint. */

/* Runs nsteps substeps exactly as mpm_step (no sorting) from the current
 * state, saving the particle state every ckpt_every substeps on the device
 * (on a mixed handle: the FP64 copy of the mixed state); force_hist (may be
 * NULL) receives nsteps x 3 forces. The state advances. */
int  mpm_adjoint_forward(mpm_handle* h, int nsteps, int ckpt_every, double* force_hist);
/* Reverse sweep of the last mpm_adjoint_forward: each segment is recomputed
 * from its checkpoint, then reversed substep by substep. dL_dforce: nsteps x 3
 * (dL/d force of each substep). dL_dcohesion (n doubles, may be NULL) and
 * *dL_dE (may be NULL) receive the gradients; the cohesion gradient is per
 * particle in the handle's current order (mpm_download_ids maps it). */
int  mpm_adjoint_backward(mpm_handle* h, const double* dL_dforce, double* dL_dcohesion, double* dL_dE);
/* Adjoints of the initial particle state after mpm_adjoint_backward: 25 rows
 * [x(3), v(3), C(9), F(9), Jp_inv] of row stride pitch >= n. */
int  mpm_adjoint_state(mpm_handle* h, double* adj, unsigned pitch);
/* Both sweeps in one call for a loss linear in the force history (dL_dforce
 * known before the run): mpm_adjoint_forward(h, nsteps, ckpt_every, NULL)
 * then mpm_adjoint_backward(h, dL_dforce, dL_dcohesion, dL_dE). */
int  mpm_adjoint(mpm_handle* h, int nsteps, int ckpt_every, const double* dL_dforce, double* dL_dcohesion,
                 double* dL_dE);

/* No counterpart in the reference. The stable cell-key sort of mpm_sort
 * (same keys, same permutation) for callers that must not have the library
 * allocate device memory: programs that plan and own every byte of the GPU
 * (their own pool or a fixed footprint), and loops that cannot take the
 * latency and device-wide synchronisation of a cudaMalloc mid-run. The
 * caller passes device pointers: soa (28 rows of `pitch` doubles, the
 * HostSideSOA row layout, n particles) and perm (n unsigned); perm receives
 * the source index of each kept particle in sorted order and *kept (host)
 * their count, disabled particles dropped. The call allocates nothing: its
 * scratch is a fixed array of about 10 MB compiled into the library, held by
 * every GPU that loads it until the process exits, which limits a call to
 * n <= 524,288 particles and (GridXTotal + 2*GridHaloSize + 1)*GridY*GridZ + 1
 * <= 1,048,576 cell keys (MPM_ERR_NOALLOC_LIMIT beyond, checked before any
 * device work). The first call on a device looks up that array's device
 * address there (with the device current) and keeps it for the life of the
 * process: make that first call before any stream capture, and make no call
 * after a cudaDeviceReset of that device or from a context other than the
 * device's primary context (the kept address then belongs to a context that
 * no longer exists or is not current). Work is issued on `stream` (a
 * cudaStream_t, NULL = legacy default) on the current device, and the call
 * waits for it. All calls share the one array: calls that overlap on the GPU
 * (other host threads, other streams) race and must be serialised by the
 * caller. Returns 0; MPM_ERR_SORT_RANGE (107) if a particle's cell key falls
 * outside the grid, in which case the contents of perm and *kept are
 * unspecified and must not be used (the next call clears the error and
 * sorts normally); or another error code. */
int  mpm_sort_permutation_noalloc(const SimParams3D* prms, const double* soa, unsigned pitch,
                                  unsigned n, unsigned* perm, unsigned* kept, void* stream);
/* Text of the last CUDA failure seen by this thread (MPM_ERR_CUDA). */
const char* mpm_last_error_string(void);

#ifdef __cplusplus
}
#endif

#endif /* ICEMPM_B200_H */
