/*
 * zf.h — C ABI of the B200-native Zebraflow coupled LBM–IB–RBC time step.
 *
 * The reference (SweSoe/Zebraflow) has no plugin or FFI boundary: its steps are
 * inline blocks of main() in ZebraflowWT.c, named only by the unused prototypes
 * at ZebraflowWT.c:163-169 and by section comments.  Every entry point below
 * replaces one of those blocks and says which one (file:line, reference paths
 * relative to the reference project root).  All state the reference keeps in
 * global static arrays (ZebraflowWT.c:171-276) lives in a zf_ctx; host buffers
 * are caller-owned and copied in or out; device memory is owned by the context.
 *
 * Conventions shared by every call:
 *  - Lattice points are addressed (i,j,k), 0-based, i in [0,nx), k fastest in
 *    dense host arrays (C order of a [nx][ny][nz] array), so B_index[i][j][k]
 *    of the reference maps to b_index[(i*ny + j)*nz + k] with i,j,k shifted by 1.
 *  - "Listed nodes" are the lattice points with B_index >= 0, enumerated in the
 *    reference's DOMLIST order (LBM_DOM_SETUP, ZebraflowWT.c:1481-1502: i outer,
 *    j, k inner).  Every per-node host array is indexed by that 0-based order.
 *  - Populations use the reference's direction order (ZebraflowWT.c:2471-2497):
 *    slot q=0..18 is the reference's c=q+1 (c=19, slot 18, is the rest
 *    population).  Population host arrays are [19][n_listed] (c-major, as F[c][l]).
 *  - Membrane, nucleus and wall-mesh coordinates are in micrometres and
 *    membrane forces in newtons, exactly as in the reference.
 *  - Every call returns ZF_OK or an error code; zf_last_error() gives a message.
 *  - One zf_ctx per host thread.  Calls enqueue on the context's CUDA stream and
 *    are ordered; zf_sync() waits for them.
 */
#ifndef ZF_H
#define ZF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZF_Q 19

enum zf_status_code {
  ZF_OK = 0,
  ZF_ERR_CUDA = 1,      /* a CUDA runtime call failed (message in zf_last_error) */
  ZF_ERR_ARG = 2,       /* invalid argument or unsupported input code */
  ZF_ERR_OVERFLOW = 3,  /* a fixed-capacity list overflowed (cell list, neighbour list) */
  ZF_ERR_NONFINITE = 4, /* non-finite value detected in a checked buffer */
  ZF_ERR_STATE = 5,     /* call made before the state it needs was set */
  ZF_ERR_NOMEM = 6      /* device allocation failed */
};

/* Wall treatment of the LBM step. */
enum zf_wall_mode {
  ZF_WALL_HALFWAY_BB = 0, /* link bounce-back halfway between fluid and non-fluid points */
  ZF_WALL_REF_EQ = 1      /* reference: wall points (B_index==0) hold feq(rho_neighbour, u=0),
                             ZebraflowWT.c:6290-6315 and :6429-6432 */
};

/* Storage type of the populations in HBM. */
enum zf_storage {
  ZF_STORE_F32 = 0,     /* plain fp32 populations f_q, as the reference stores F */
  ZF_STORE_F16 = 1,     /* fp16 of S*(f_q/w_q - rho_ref), arithmetic in fp32 */
  ZF_STORE_BF16 = 2,    /* bf16 of the same deviation */
  ZF_STORE_F32_DEV = 3  /* fp32 of the deviation f_q/w_q - rho_ref */
};

/* Run-time parameters.  zf_params_default() fills the reference's values
 * (ZebraflowWT.c:34-161) so that a default-filled struct reproduces the
 * reference constants; callers override lattice size and what they need. */
typedef struct zf_params {
  /* lattice */
  int32_t nx, ny, nz;       /* lattice box (reference IM, JM, KM) */
  double origin[3];         /* um, coordinates of lattice point (0,0,0) (reference X0,Y0,Z0) */
  double dx;                /* um, lattice spacing (reference DX = 0.5) */
  double dt;                /* us, time step (reference DT = 0.5); also the factor that
                               multiplies BODYFORCE in the Guo step, ZebraflowWT.c:6133,6141 */
  float tau;                /* BGK relaxation time of every fluid point */
  int32_t tau_from_phase;   /* 1: tau = 0.5 + 0.72*B_index per point (ZebraflowWT.c:6110) */
  float g[3];               /* uniform effective Guo body force, lattice units; added to
                               dt*BODYFORCE (0 in the reference) */
  int32_t wall_mode;        /* enum zf_wall_mode */
  int32_t periodic[3];      /* 1: the axis wraps (the reference wraps none) */
  int32_t storage;          /* enum zf_storage */
  float rho_ref;            /* reference density of the deviation storage */
  /* membrane / IB / coupling (SI units unless stated) */
  int32_t stagger;          /* membrane + IB solver every `stagger` LBM steps (SOLVERSTAGGER=50) */
  double Es;                /* membrane shear modulus, N/m (reference 3e-6) */
  double Es_nucleus_ratio;  /* nucleus shear modulus / Es (reference 0.1, ZebraflowWT.c:2039) */
  double kbend;             /* bending coefficient, J (reference 1.3856406e-19) */
  double kd;                /* local area coefficient, N/m (reference 3.6e-5) */
  double ka;                /* global area coefficient, N/m (reference 7.7e-5) */
  double kv;                /* volume coefficient, N/m^2 (reference 55) */
  double area0;             /* rest cell area, m^2; <= 0: from the rest mesh (reference RBC_SURF) */
  double volume0;           /* rest cell volume, m^3; <= 0: from the rest mesh (reference MCV) */
  double kT;                /* TEMPERATURE*BOLTZ, J */
  double e_ratio_eq;        /* rest / maximum spectrin length (0.3154574132) */
  int32_t calib_passes;     /* fixed-point passes of the spring calibration (51) */
  double gamma_p;           /* repulsion-to-force coefficient of IB spreading (1e-7) */
  double unit_mass;         /* kg, lattice mass unit (UNITMASS = 1.25e-15) */
  double bforce_scale;      /* LBM_BFORCE_SCALE = (1/3)*dx/dt^2 in SI (6.6667e5) */
  double vel_scale;         /* VEL_SCALE (1.0) */
  double vmax_remove;       /* node speed that removes a cell (5e-3) */
  int32_t remove_count;     /* screened-term count that removes a cell (500) */
  int32_t nuc_list_period;  /* nucleus-membrane list rebuild period in iterations (1000) */
  int32_t nuc_list_max;     /* capacity of each nucleus node's triangle list (NucMembMAX) */
  int32_t stochastic_round; /* 16-bit storage forms: 1 = hardware stochastic rounding
                               (cvt.rs, hashed random bits per point, step and direction),
                               0 = round to nearest */
  int32_t wall_list_max;    /* capacity of a wall node's triangle list (reference 12) */
} zf_params;

typedef struct zf_ctx zf_ctx;

/* Counters returned by zf_get_status (reference: printf + simfailure, which
 * is counted but never read, ZebraflowWT.c:5647, :7086-7345). */
typedef struct zf_status {
  int64_t screened_terms;   /* force terms dropped as NaN/inf/over 1e-10 N */
  int64_t cells_removed;    /* cells removed (bad geometry or speed) */
  int64_t list_overflows;   /* cell-list / nucleus-list entries that did not fit */
  int64_t bc_no_neighbour;  /* wall points without a designated neighbour */
  int64_t iter;             /* completed LBM iterations */
} zf_status;

/* ---- context ------------------------------------------------------------ */

/* Reference constants (ZebraflowWT.c:34-161) into *p. */
void zf_params_default(zf_params* p);

/* sizeof(zf_params), so that bindings can check their struct layout. */
size_t zf_params_size(void);

/* Creates a context on CUDA device `device`; params are copied.  Replaces the
 * global state of ZebraflowWT.c:171-276.  Returns NULL on failure
 * (zf_last_error says why). */
zf_ctx* zf_create(const zf_params* p, int device);
void zf_destroy(zf_ctx* ctx);
const char* zf_last_error(void);
int zf_sync(zf_ctx* ctx);
int zf_get_status(zf_ctx* ctx, zf_status* out);

/* ---- lattice ------------------------------------------------------------- */

/* Sets the lattice from reference B_index codes ([nx][ny][nz], k fastest):
 * <0 solid, 0 wall point, 1..9 fluid of that phase, 1001..1009 pressure
 * inlet/outlet points of the reference's waveforms (ZebraflowWT.c:6316-6426;
 * reference wall mode only: they take feq(P(t)/LBM_PRESSURE_SCALE + 1, u) of
 * their designated neighbour every step).  Other codes (the deprecated 4998)
 * are rejected with ZF_ERR_ARG.
 * Builds the listed-node order (LBM_DOM_SETUP, ZebraflowWT.c:1481-1502), the
 * designated neighbour of every wall point (LBM_BC_SETUP, ZebraflowWT.c:1506-1589)
 * and the device tile index; initialises f = feq(rho_ref, 0) (ZebraflowWT.c:5253-5295). */
int zf_set_lattice(zf_ctx* ctx, const int32_t* b_index);

/* Number of listed nodes (reference DOMMAX) and of fluid nodes (1..9). */
int zf_num_listed(zf_ctx* ctx, int64_t* n_listed, int64_t* n_fluid);

/* Listed-node coordinates in DOMLIST order, [n_listed][3] (i,j,k), 0-based. */
int zf_get_domlist(zf_ctx* ctx, int32_t* ijk);

/* ---- fluid fields (reference F, D/U/V/W, BODYFORCE; ZebraflowWT.c:176-183) -- */

/* f: [19][n_listed] populations; NULL keeps them.  The stored moments
 * D,U,V,W become those of the uploaded populations (the reference's restart
 * loads both, ZebraflowWT.c:2649-2700). */
int zf_upload_populations(zf_ctx* ctx, const float* f);
int zf_download_populations(zf_ctx* ctx, float* f);
/* bodyforce: [3][n_listed], reference BODYFORCE units (IB force density) */
int zf_upload_bodyforce(zf_ctx* ctx, const float* bodyforce);
int zf_download_bodyforce(zf_ctx* ctx, float* bodyforce);
/* D,U,V,W [n_listed] written by the last LBM step that stored moments
 * (post-collision moments without force shift, ZebraflowWT.c:6599-6616). */
int zf_download_moments(zf_ctx* ctx, float* D, float* U, float* V, float* W);

/* Recomputes the stored D,U,V,W from the current populations (the moments
 * of the reference's LBM_FLUID pass, ZebraflowWT.c:6603-6616), so that a
 * snapshot can be taken after any step. */
int zf_lbm_moments(zf_ctx* ctx);

/* ---- LBM step ------------------------------------------------------------ */

/* One LBM time step: pull stream + BGK/Guo collision (ZebraflowWT.c:6100-6145),
 * wall treatment (:6290-6315, :6429-6432 in ZF_WALL_REF_EQ; bounce-back links
 * in ZF_WALL_HALFWAY_BB) and the moments/copy pass (:6599-6626), fused into one
 * kernel over the tile index with ping-pong buffers.  store_moments=1 writes
 * D,U,V,W (post-collision, as :6611-6614); zero_bodyforce=1 clears BODYFORCE
 * after it was used (:6622-6624). */
int zf_lbm_step(zf_ctx* ctx, int store_moments, int zero_bodyforce);

/* n LBM steps back to back (moments stored on the last one only). */
int zf_lbm_steps(zf_ctx* ctx, int n);

/* One LBM step that also returns the global mass: the FP64 sum of the
 * pre-collision density over fluid points, reduced inside the step kernel
 * (per-block partial sums, then a fixed-order sum), copied to *mass. */
int zf_lbm_step_mass(zf_ctx* ctx, int store_moments, int zero_bodyforce, double* mass);

/* No counterpart in the reference.  zf_lbm_step_mass for callers that cannot
 * call cudaMalloc once their run has started (device memory owned by another
 * allocator that has already reserved the GPU; loops that must not take
 * cudaMalloc's implicit device synchronisation or an out-of-memory failure
 * mid-run): it allocates nothing.  Its reduction scratch is a file-scope
 * device array of 65,536 + 1 doubles (512 KB, held on every GPU that loads the
 * library until exit), so it serves lattices of at most 65,536 blocks of four
 * 4x4x4 tiles with fluid (262,144 tiles); larger ones get ZF_ERR_ARG with a
 * message.  The first call on a device does the set-up: it looks the array's
 * address up (cudaGetSymbolAddress) and, with lazy module loading, may load the
 * library's device code, which is when the array's 512 KB are reserved; make
 * that first call once, as a warm-up, before the caller's allocator takes the
 * GPU and before any stream capture.  The address is cached per device for the
 * primary context: do not call this again on a device after cudaDeviceReset.
 * Every call overwrites the scratch, so nothing carries over between calls;
 * calls that overlap on the GPU (other streams or contexts of the same device)
 * share the scratch and race. */
int zf_lbm_step_mass_noalloc(zf_ctx* ctx, int store_moments, int zero_bodyforce, double* mass);

/* Z-slab halo exchange (no counterpart in the reference, which runs on one
 * node).  A lattice cut into z slabs, one per GPU, each with one 4-plane tile
 * layer of halo on either side, stays exact if after every step the halo
 * plane next to each face receives, from the rank owning it, the populations
 * the interior pulls across that face: those of the 5 directions with
 * e_z = dir (+1: pulled upwards, -1: downwards) of the listed points of one
 * plane.  zf_plane_count gives the number of listed points of plane z = k of
 * this context's lattice; zf_plane_pack copies their dir-populations of the
 * current state, in (x, y) order, into dev_buf ([n][5] storage elements: 4
 * bytes each for the fp32 forms, 2 for fp16/bf16; device memory, written on
 * the context's stream); zf_plane_unpack writes such a buffer into plane k. */
/* No counterpart in the reference.  Slab stepping: a context holding a z slab
 * with one tile layer (4 planes) of halo on either side declares its interior
 * planes [k_lo, k_hi) (multiples of 4); its active tiles then split into the
 * inner tile layers and the two face layers next to the halo, and the halo
 * layers are not stepped.  zf_lbm_step_part(ctx, 0, 0) steps the inner layers,
 * which read no halo plane, so it can run while the halo exchange of the
 * previous step is in flight; zf_lbm_step_part(ctx, 1, 1) steps the face
 * layers once the halo planes are unpacked and completes the step (wall pass,
 * buffer swap, iteration count).  Neither stores moments or clears BODYFORCE. */
int zf_set_slab(zf_ctx* ctx, int k_lo, int k_hi);
int zf_lbm_step_part(zf_ctx* ctx, int part, int finish);

int zf_plane_count(zf_ctx* ctx, int k, int32_t* n);
int zf_plane_pack(zf_ctx* ctx, int k, int dir, void* dev_buf);
int zf_plane_unpack(zf_ctx* ctx, int k, int dir, const void* dev_buf);

/* Sets the uniform effective body force g (lattice units) used from the next step. */
int zf_set_uniform_force(zf_ctx* ctx, const float* g3);

/* Runs subsequent work of the context on `cuda_stream` (a cudaStream_t of the
 * context's device, e.g. the current PyTorch stream); NULL restores the
 * context's own stream.  Work already queued is not moved. */
int zf_set_stream(zf_ctx* ctx, void* cuda_stream);

/* Total mass sum_l sum_q f (FP64 reduction over fluid points, or all listed
 * points when include_walls=1). */
int zf_mass(zf_ctx* ctx, int include_walls, double* mass);

/* Device time of the last `n` LBM steps run by zf_lbm_steps_timed, in ms,
 * measured with CUDA events on the context stream. */
int zf_lbm_steps_timed(zf_ctx* ctx, int n, float* ms);

/* Bytes of device memory the context holds. */
int zf_device_bytes(zf_ctx* ctx, int64_t* bytes);

/* ---- membrane mesh and cells ---------------------------------------------- */

/* Sets the membrane mesh shared by every cell and its nucleus mesh, with the
 * rest shapes the springs are calibrated on (the reference reads them from
 * ZFISHRBCNODES.dat / ZFISHRBCTRIANGLES.dat / NucleusNodes.dat /
 * NucleusEdges.dat, ZebraflowWT.c:1601-1922).  tri: [n_tri][3] 1-based,
 * counter-clockwise seen from outside; rest: [n_node][3] um; edge_n:
 * [n_edge_n][2] 1-based; rest_n: [n_node_n][3] um.  Builds the edge/rhombus
 * list in the reference's order (CGSM_ZFISHRBC_DATA_GEN, ZebraflowWT.c:1640-1805),
 * calibrates WLC/POW springs (CGSM_FILAMENT_PARAMETERS, :1930-2053, iterated
 * as :2339-2346), rest metrics (CGSM_EQUILIBRIUM_METRICS, :2056-2223) and rest
 * triangle areas (:2387-2460).  Cells set before are dropped. */
int zf_set_mesh(zf_ctx* ctx, int n_node, int n_tri, const int32_t* tri, const double* rest,
                int n_node_n, int n_edge_n, const int32_t* edge_n, const double* rest_n);

/* Number of membrane edges and the rest cell area (m^2) / volume (m^3) used
 * by the global-area and volume constraints. */
int zf_mesh_info(zf_ctx* ctx, int32_t* n_edge, double* area0, double* volume0);

/* Edge list [n_edge][6] (n1,n2,n3,n4,tri1,tri2, 1-based: EDGENODE_LIST[edge][1..6],
 * ZebraflowWT.c:224) and per edge the first-visitor flags of the area/volume
 * terms (bit 0: tri1, bit 1: tri2; AREA_UPDATE, :7127-7128).  NULL skips. */
int zf_get_edges(zf_ctx* ctx, int32_t* edges, uint8_t* area_first);

/* Spring and rest parameters: epar [5][n_edge] = LMAX, Plength, kp,
 * SINETHETA0, COSINETHETA0 (ZebraflowWT.c:228); epar_n [3][n_edge_n] =
 * LMAX_N, Plength_N, kp_N (:235); tri_area_eq [n_tri] (TRI_AREA_eq, :220). */
int zf_get_edge_params(zf_ctx* ctx, float* epar, float* epar_n, float* tri_area_eq);

/* Places n_cells cells: x [3][n_cells][n_node] and xn [3][n_cells][n_node_n]
 * in um (NODECOORD / NODECOORD_N layout, ZebraflowWT.c:225, :238).  All cells
 * start independent (reference CellStatus 1). */
int zf_set_cells(zf_ctx* ctx, int n_cells, const double* x, const double* xn);

/* Positions (layouts as zf_set_cells) and status per cell (1 active,
 * -5000 removed).  NULL skips. */
int zf_get_cells(zf_ctx* ctx, double* x, double* xn, int32_t* status);

/* No counterpart in the reference.  zf_get_cells without waiting: the copies
 * of the positions and statuses as they stand after the work queued so far
 * run on a second stream while the caller queues more steps; the next kernel
 * that changes positions or statuses (the membrane forces and the position
 * update of the next membrane iteration, zf_set_cells, zf_load_state) waits
 * for them, so the LBM iterations in between overlap the copy.  The host
 * buffers must be pinned (cudaHostAlloc / cudaHostRegister) for the copy to
 * run asynchronously, and hold their values once zf_wait_cells returns. */
int zf_get_cells_async(zf_ctx* ctx, double* x, double* xn, int32_t* status);
int zf_wait_cells(zf_ctx* ctx);

/* F_Total [3][n_cells][n_node] and F_Total_N [3][n_cells][n_node_n] in N. */
int zf_get_cell_forces(zf_ctx* ctx, float* ftot, float* ftot_n);

/* NODE_VEL / NODE_VEL_N (um/us, fp64) and NODE_WALLREPUL / NODE_WALLREPUL_N
 * (velocity increments) of the last membrane step. */
int zf_get_cell_kinematics(zf_ctx* ctx, double* vel, double* vel_n, float* wrep, float* wrep_n);

/* Geometry of the last membrane step: TRI_AREA [n_cells][n_tri] (m^2),
 * TRI_NORMAL and TRI_CENTROID [3][n_cells][n_tri], NODE_NORMAL
 * [3][n_cells][n_node], and per cell [n_cells][8]: area (m^2), volume (m^3),
 * centroid (um, 3), F_AREA_GLOBAL, F_VOLUME_SCALAR, unused. */
int zf_get_cell_geometry(zf_ctx* ctx, float* tri_area, float* tri_normal, float* tri_centroid,
                         float* node_normal, float* cell_f);

/* Membrane and nucleus forces of every cell (one CTA per cell): force
 * reset (ZebraflowWT.c:5704-5745), triangle geometry and sliver repulsion
 * (CGSM_AREA, :5749-6096), cell area and centroid (:6717-6796),
 * CGSM_LOCAL_FORCES (:6800-7386), nucleus springs (:7388-7471), bad-cell
 * removal (:7473-7501) and CGSM_VOLUME_CALC (:7510-7535).  Writes F_Total,
 * F_Total_N and the geometry; clears node velocities and repulsions. */
int zf_cgsm_forces(zf_ctx* ctx);

/* ---- vessel wall and the IB coupling ------------------------------------ */

/* Sets the lumen wall mesh: xyz [3][n_node_w] (um, WALLNODECOORD), tri
 * [3][n_tri_w] 1-based node ids (WALLCELLNODE after its +1, ZebraflowWT.c:3840-3852),
 * normals [3][n_tri_w] pointing into the lumen (WALLCELLNORMALS).  Builds the
 * nearest-wall-node index of every lattice point within +-4 points of a wall
 * node (W_index, :3715-3822), the node-to-triangle lists (:3899-3935, capacity
 * zf_params.wall_list_max), triangle centroids (:4648-4663) and the void
 * velocity of non-fluid points near the wall (:4788-4852). */
int zf_set_wall(zf_ctx* ctx, int n_node_w, const float* xyz, int n_tri_w, const int32_t* tri,
                const float* normals);

/* W_index (1-based wall node, 0 none) and void velocity [3] of every lattice
 * point as dense [nx][ny][nz] arrays (NULL skips). */
int zf_get_wall_index(zf_ctx* ctx, int32_t* windex, float* uvoid);

/* IB velocity interpolation of every membrane and nucleus node from the
 * moments of the last LBM step run with store_moments=1, plus the nearest
 * wall triangle search and wall repulsion (ZebraflowWT.c:8690-9142,
 * :9149-9430).  Adds to NODE_VEL / NODE_VEL_N and NODE_WALLREPUL. */
int zf_ibm_interp(zf_ctx* ctx);

/* Number of triangle centroids the cell list of the last membrane step holds
 * at each listed point, DOMLIST order (the reference's EulNeigh[0][o], filled
 * by CGSM_AREA, ZebraflowWT.c:5857-5900); 0 before any membrane step. */
int zf_get_cell_list_counts(zf_ctx* ctx, int32_t* counts);

/* Nucleus-membrane repulsion (ZebraflowWT.c:9516-9730); rebuild_lists=1
 * rebuilds every nucleus node's triangle list (the reference does so every
 * 1000 iterations, :9527).  Adds to NODE_WALLREPUL. */
int zf_nuc_memb_repulsion(zf_ctx* ctx, int rebuild_lists);

/* Builds the triangle cell list (EulNeigh, ZebraflowWT.c:5857-5902) and adds
 * the membrane-membrane repulsion to NODE_WALLREPUL (:9911-10053). */
int zf_rbc_rbc_repulsion(zf_ctx* ctx);

/* IB spreading of F_Total + gamma_p*NODE_WALLREPUL into BODYFORCE, after
 * NODE_VEL += NODE_WALLREPUL (ZebraflowWT.c:10737-10870, :10874-10990). */
int zf_ibm_spread(zf_ctx* ctx);

/* x += NODE_VEL*DT*SOLVERSTAGGER for membrane and nucleus nodes; a cell
 * with a node faster than vmax_remove (or not finite) is removed
 * (ZebraflowWT.c:11965-12031). */
int zf_update_positions(zf_ctx* ctx);

/* Wall shear stress and wall pressure at the wall-mesh nodes, as the
 * reference's post-processor computes them (PostProWSSandPressure.c:275-369)
 * from the current populations (post-collision moments, :6603-6616):
 *   probe x_m + DX n_m, velocity interpolated there with the Peskin cosine
 *   weights inside 2 DX over fluid points (B_index 1..9) of the +-3 window,
 *   WSS = -0.0012 Pa.s * (u - (u.n) n) / (DX 1e-6 m)   [wss: [3][nw], Pa];
 *   pressure (D-1)/3*1e4 - pgauge at the nearest listed point within
 *   1.42 DX of x_m                                    [pressure: [nw], Pa];
 *   valid = 0 where no such point exists or the pressure is below 1 Pa.
 * node_normals [3][nw] are unit normals into the lumen; NULL takes the
 * area-weighted mean of the wall triangles' normals at each node.  With a
 * periodic z axis the windows wrap (the reference has no periodic axis).
 * pressure and valid may be NULL.  Waits for the result. */
int zf_wss(zf_ctx* ctx, const float* node_normals, double pgauge, float* wss, float* pressure,
           int32_t* valid);

/* Wall-shear-stress objective and its hand-written adjoint (no counterpart
 * in the reference, which has no adjoint; the objective uses its WSS,
 * PostProWSSandPressure.c:319-369).  The forward that is differentiated
 * starts from the context's current populations, with the cells held at their
 * current positions:
 *   BODYFORCE = S(x) F_total(x; Es, kb) + fb       (spread membrane forces,
 *                                                   ZebraflowWT.c:10737-10990)
 *   nsteps LBM steps (:6100-6145) with that BODYFORCE, tau and g;
 *   J = mean over steps t0..t1 (1 <= t0 <= t1 <= nsteps) of the mean over the
 *       patch's wall nodes of |WSS| (Pa) of the state after step t.
 * fb: [3][n_listed] per-node body-force field (DOMLIST order) or NULL (zero).
 * node_normals as in zf_wss.  Needs halfway bounce-back and a uniform tau;
 * with fp16/bf16 population storage the forward runs in that storage and the
 * adjoint (fp32) treats its rounding as the identity.  Both calls leave the
 * populations and BODYFORCE as they were.
 * zf_wss_adjoint keeps the populations of every checkpoint_interval-th step,
 * recomputes each interval backwards from them, and returns J and
 * dJ/dfb ([3][n_listed], the same as dJ/dBODYFORCE), dJ/dtau, dJ/dEs and
 * dJ/dkb (membrane shear and bending moduli, through the spread forces at
 * the held positions; 0 without cells).  Any output may be NULL. */
int zf_wss_objective(zf_ctx* ctx, int nsteps, int t0, int t1, const int32_t* patch, int n_patch,
                     const float* node_normals, const float* fb, double* J);
int zf_wss_adjoint(zf_ctx* ctx, int nsteps, int t0, int t1, const int32_t* patch, int n_patch,
                   const float* node_normals, const float* fb, int checkpoint_interval, double* J,
                   float* dJ_dfb, double* dJ_dtau, double* dJ_dEs, double* dJ_dkb);

/* Flux-split objective and its adjoint (no counterpart in the reference): the
 * same differentiated forward as zf_wss_objective, with
 *   J = mean over steps t0..t1 of Q_0 / (Q_0 + Q_1),
 *   Q_s = sum over the listed points pts_s (DOMLIST indices, 0-based, fluid
 *         points, the two sets disjoint) of U . nrm_s,
 * U the post-collision velocity (moments without force shift, as the
 * reference's U, V, W, ZebraflowWT.c:6611-6614).  For two outlet
 * cross-sections J is the share of the flow leaving through the first.
 * Outputs as zf_wss_adjoint; the wall mesh is not needed. */
int zf_flux_objective(zf_ctx* ctx, int nsteps, int t0, int t1, const int32_t* pts0, int n0, const float* nrm0,
                      const int32_t* pts1, int n1, const float* nrm1, const float* fb, double* J);
int zf_flux_adjoint(zf_ctx* ctx, int nsteps, int t0, int t1, const int32_t* pts0, int n0, const float* nrm0,
                    const int32_t* pts1, int n1, const float* nrm1, const float* fb, int checkpoint_interval,
                    double* J, float* dJ_dfb, double* dJ_dtau, double* dJ_dEs, double* dJ_dkb);

/* The forward the four calls above differentiate.  move = 0 (the default):
 * the cells stay at their positions over the window.  move = 1: the cells
 * move -- the window is the reference time loop (zf_step, ZebraflowWT.c:
 * 5646-12190) from the context's iteration, with BF_0 = S(x_0) F(x_0) + fb
 * in effect until the first membrane iteration and fb added to every spread
 * field; the adjoint carries the positions' adjoint through the position
 * update (:11965-11997), interpolation (:8963-8996), spreading (:10745-10870)
 * and the membrane and nucleus forces (:5749-7535), and holds the repulsion
 * velocities through the wall, nucleus-membrane and RBC-RBC repulsions
 * (:9055-9077, :9516-9730, :9919-10053; their choices of wall triangle, list
 * entries and facing triangles are held, as the derivative of the branch the
 * forward took).  Memory: positions, spread forces and the
 * spread field of every membrane iteration in the window are kept.  The calls
 * leave the cells' positions, statuses, counters and nucleus-membrane lists
 * as they were. */
int zf_adjoint_move_cells(zf_ctx* ctx, int move);

/* dJ/dx_0 and dJ/dxn_0 ([3][cells][nodes], um^-1 per unit of J) of the last
 * adjoint run with moving cells, with respect to the positions the window
 * started from. */
int zf_adjoint_position_gradient(zf_ctx* ctx, float* dJ_dx, float* dJ_dxn);

/* Vector-Jacobian product of the membrane and nucleus forces at the current
 * positions (ZebraflowWT.c:5749-7535): given lam ([3][cells][nn], the weights
 * of the membrane node forces) and lam_n ([3][cells][nnn] or NULL), returns
 * dx = lam^T dF/dx, dxn = lam_n^T dF/dxn, and lam^T dF/dEs, lam^T dF/dkb.
 * Any output may be NULL. */
int zf_membrane_vjp(zf_ctx* ctx, const float* lam, const float* lam_n, float* dx, float* dxn, double* dEs,
                    double* dkb);

/* Vector-Jacobian product of the repulsion velocities (NODE_WALLREPUL) of a
 * membrane iteration at the current positions: the wall repulsion
 * (ZebraflowWT.c:9055-9077, with the nucleus nodes' share, :9415-9430), the
 * nucleus-membrane repulsion (:9516-9730, lists rebuilt at the current
 * positions) and the RBC-RBC repulsion (:9919-10053): given lam_w
 * ([3][cells][nn], the weights of the membrane nodes' repulsion velocities),
 * returns dx = lam_w^T dwrep/dx and dxn = lam_w^T dwrep/dxn.  Overwrites the
 * cells' forces, velocities and repulsion velocities, as a membrane iteration
 * would. */
int zf_repulsion_vjp(zf_ctx* ctx, const float* lam_w, float* dx, float* dxn);

/* The coupled step on a lattice split into z slabs (one context per slab, no
 * counterpart in the reference).  The context's lattice is its slab with
 * halo planes, not periodic in z; every context holds all cells (positions in
 * the global frame), the wall mesh with its z folded into the frame
 * [origin z, origin z + lz), and:
 *   zf_set_ib_slab: the planes [k_lo, k_hi) this slab owns (at least 8 halo
 *     planes on either side) and the period lz (um) of the whole lattice along
 *     z.  Interpolation then sums over owned planes only, spreading writes
 *     owned planes only, and the wall, nucleus-membrane and RBC-RBC repulsions
 *     run for the nodes whose lattice index lies in the owned planes.
 *   zf_cells_reduce_size / zf_cells_reduce_buffer: the node velocities and
 *     repulsion velocities as one fp64 device buffer of n values (dir 0:
 *     copied into it, 1: back).  Summed over the slabs after the repulsions
 *     and before spreading, it gives every slab the unsplit values.
 *   zf_lbm_step_part_mf: zf_lbm_step_part with the moment store and body-force
 *     clearing of a membrane iteration. */
int zf_set_ib_slab(zf_ctx* ctx, int k_lo, int k_hi, double lz);
int zf_cells_reduce_size(zf_ctx* ctx, int64_t* n);
int zf_cells_reduce_buffer(zf_ctx* ctx, int dir, void* dev_buf);
int zf_lbm_step_part_mf(zf_ctx* ctx, int part, int finish, int store_moments, int zero_bodyforce);

/* Periodic parent segments and cell cloning (the reference's inflow,
 * ZebraflowWT.c:11926-11960, :12193-12403), as host steps on host arrays
 * between membrane iterations; zebraflow_b200/inflow.py drives them around a
 * parent-segment context and a region context.  A segment is periodic over
 * [z0, z1) (um); direction +1: the flow leaves it at z1, -1: at z0; dx is the
 * lattice spacing (um).  Statuses as the reference's (:256-263): parents 2
 * (interior) or 4 (cloned, not yet re-armed); region slots -(p + 1) (clone
 * slaved to parent p), 1 (independent), -5000 (free).
 *   zf_inflow_slaves: after the region's update, the nodes of slaved clones
 *     that were not yet 5 dx past the exit plane move with their parent's
 *     node velocity (vp, vnp) instead of their own (vr, vnr; x += (vp - vr)
 *     dt_stagger); a clone whose nodes all passed the plane becomes 1.
 *   zf_inflow_parents: after the segment's update, the parents' z folded into
 *     [z0, z1); clone[p] = 1 for a status-2 parent that crossed the exit plane
 *     and has not regressed; status-4 parents are re-armed inside the window.
 *   zf_inflow_clone: every parent with clone[p] copied, in order, into the
 *     first free slot (z made contiguous across the exit plane), the slot
 *     -(p + 1), the parent 4; cloned_into[p] the slot or -1 (may be NULL). */
typedef struct {
  double z0, z1;
  int32_t direction;
  double dx;
} zf_inflow_segment;
int zf_inflow_slaves(const zf_inflow_segment* seg, double dt_stagger, int n_slots, int nn, int nnn, double* xr,
                     double* xnr, const double* vr, const double* vnr, int32_t* status_r, int n_parents,
                     const double* vp, const double* vnp);
int zf_inflow_parents(const zf_inflow_segment* seg, int n_parents, int nn, int nnn, double* x, double* xn,
                      int32_t* status, int32_t* regress, int32_t* clone);
int zf_inflow_clone(const zf_inflow_segment* seg, int n_parents, int nn, int nnn, const double* xp,
                    const double* xnp, int32_t* status_p, int32_t* regress_p, int32_t* clone, int n_slots,
                    double* xr, double* xnr, int32_t* status_r, int32_t* cloned_into);

/* The cells' positions and statuses overwritten from host arrays of the
 * context's cell count (zf_set_cells keeps the cell count and buffers but
 * makes every cell active; these keep everything else): x [3][cells][nn],
 * xn [3][cells][nnn] (or NULL), status [cells] (or NULL; -5000 a free slot,
 * skipped by every kernel, > 0 active). */
int zf_put_cells(zf_ctx* ctx, const double* x, const double* xn, const int32_t* status);

/* nsteps iterations of the reference time loop (ZebraflowWT.c:5646-12190):
 * every iteration an LBM step; every `stagger`-th iteration also the
 * membrane forces, IB interpolation, repulsions, spreading and position
 * update, in the reference's order. */
int zf_step(zf_ctx* ctx, int nsteps);

/* zf_step timed with CUDA events on the context stream (ms). */
int zf_step_timed(zf_ctx* ctx, int nsteps, float* ms);

/* One iteration of zf_step that also returns the FP64 global mass reduced
 * inside its LBM kernel (see zf_lbm_step_mass); waits for the result. */
int zf_step_mass(zf_ctx* ctx, double* mass);

/* Number of kernels the context has launched so far. */
int zf_launch_count(zf_ctx* ctx, int64_t* n);

/* Instrumentation of zf_step: with enable=1, CUDA events bracket each run of
 * consecutive plain LBM steps (the steps between membrane blocks) and each
 * membrane/IB block, up to `capacity` of each; zf_profile_read returns the
 * summed device times (ms), the number of LBM launches in the timed runs and
 * the number of membrane blocks. */
int zf_profile(zf_ctx* ctx, int enable, int capacity);
int zf_profile_read(zf_ctx* ctx, float* lbm_ms, int* lbm_count, float* membrane_ms,
                    int* membrane_count);

/* Per-stage device time (ms) of the membrane iterations profiled since
 * zf_profile(ctx, 1, ...), summed over `*blocks` iterations: stage_ms[8] =
 * {membrane forces, LBM step, IB interpolation + wall repulsion,
 *  nucleus-membrane repulsion, cell-list build, RBC-RBC repulsion,
 *  IB spreading, position update}. */
int zf_profile_stages(zf_ctx* ctx, float* stage_ms, int* blocks);

/* Completed iterations (the reference's iter). */
int zf_iteration(zf_ctx* ctx, int64_t* iter);

/* Sets the count of completed iterations, as a run restarted at iteration
 * `iter` has it: the next step is iteration iter + 1, which fixes the
 * membrane cadence, the pressure waveforms' time and the stochastic-rounding
 * seed. */
int zf_set_iteration(zf_ctx* ctx, int64_t iter);

/* Exact checkpoints (the reference restarts from its CSV snapshots, rebuilding
 * the populations as feq(D, u), ZebraflowWT.c:2649-2700, :5253-5295, which
 * leaves the trajectory).  zf_save_state writes what the next step reads: the
 * current populations in their storage form, BODYFORCE, the stored moments,
 * the cells' fp64 positions and velocities, forces, repulsion increments,
 * statuses and counters, the nucleus-membrane lists and the iteration count.
 * zf_load_state restores it into a context set up with the same lattice,
 * storage form, mesh and cell count (else ZF_ERR_ARG), after which zf_step
 * continues the saved run.  Both wait for the context's queued work. */
int zf_save_state(zf_ctx* ctx, const char* path);
int zf_load_state(zf_ctx* ctx, const char* path);

/* ---- input generators (synthetic stand-ins for the reference's input files,
 *      FLUIDdomainBindex.csv read at ZebraflowWT.c:2574-2619) ---------------- */

/* Straight tube along z in lattice units: B_index 1 for (i-cx)^2+(j-cy)^2 < R^2,
 * 0 for non-fluid points linked to a fluid point, -1 elsewhere. */
int zf_gen_tube(int nx, int ny, int nz, double cx, double cy, double R, int periodic_z,
                int32_t* b_index);

/* Z-periodic Y-bifurcation: parent radius Rp splits at +-half_angle_deg (in x)
 * into two daughters of radius Rd that run straight and merge back.  layout
 * (6 doubles, may be NULL) receives z_split, z_straight, z_converge, z_merge,
 * daughter offset. */
int zf_gen_bifurcation(int nx, int ny, int nz, double Rp, double Rd, double half_angle_deg,
                       int32_t* b_index, double* layout);

/* Unit icosphere subdivided `level` times: 10*4^level+2 nodes into xyz
 * [n][3], 20*4^level triangles into tri [n][3] (1-based, outward winding). */
int zf_gen_icosphere(int level, double* xyz, int32_t* tri);

/* Wall meshes of the generated vessels in the zf_set_wall layouts (um):
 * a cylinder of radius R (lattice units) around lattice axis (cx, cy), rings
 * every h lattice units with nseg segments; and the zero set of the
 * bifurcation's signed distance by marching tetrahedra.  Normals point into
 * the lumen.  With NULL outputs only n_node/n_tri are returned; otherwise the
 * outputs must hold cap_node / cap_tri entries per component. */
int zf_gen_wall_tube(double cx, double cy, double R, int nz, double h, int nseg,
                     const double* origin, double dx, int* n_node, int* n_tri, float* xyz,
                     int32_t* tri, float* nrm, int cap_node, int cap_tri);
int zf_gen_wall_bifurcation(int nx, int ny, int nz, double Rp, double Rd, double half_angle_deg,
                            const double* origin, double dx, int* n_node, int* n_tri, float* xyz,
                            int32_t* tri, float* nrm, int cap_node, int cap_tri);

/* Seeded cell placement (stand-in for the reference's cell start files,
 * ZebraflowWT.c:5297-5637): centres uniform over the fluid points of b
 * ([nx][ny][nz] B_index codes), orientations uniform, candidates rejected
 * when their ellipsoid (semi-axes `axes` um + margin) overlaps a placed one
 * or a membrane node has a non-fluid point in the lattice cube of half-width
 * max(1, ceil(wall_clear / dx)) around it (wall_clear in um; 0 keeps one
 * lattice unit of clearance).
 * rest [n_node][3] / rest_n [n_node_n][3] are the shapes (um) around their
 * centres; x [3][n_cells][n_node], xn [3][n_cells][n_node_n] receive um;
 * *placed the number placed (the first *placed cells are valid). */
int zf_gen_cells(const int32_t* b, int nx, int ny, int nz, const double* origin, double dx,
                 int periodic_z, int n_cells, int n_node, const double* rest, int n_node_n,
                 const double* rest_n, const double* axes, double margin, double wall_clear,
                 uint64_t seed, double* x, double* xn, int* placed);

/* ---- the reference's file formats (host only, no device needed) -----------
 * Readers of the reference's input files and writers of the snapshots its
 * OUTPUT() (ZebraflowWT.c:282-509) and post-processor write, on caller-owned
 * host arrays in the layouts above.  Writers print with the reference's
 * formats, so a file written from the same values is the reference's file
 * byte for byte.  Coordinates map to lattice points as the reference does:
 * 0-based i = (int)((x - origin)/dx + 1.01) - 1. */

/* FLUIDdomainBindex.csv (read at ZebraflowWT.c:2574-2619): a header line, then
 * "B_index,X,Y,Z" per row.  b_index [nx][ny][nz] is set to -1 (:2516) and then
 * to each row's code; a row outside the box is an error. */
int zf_read_bindex_csv(const char* path, int nx, int ny, int nz, const double* origin, double dx,
                       int32_t* b_index, int64_t* n_rows);

/* Boundary CSV of a parent segment, "Bindex","D","U","V","W","Points:0",
 * "Points:1","Points:2" (DAparentBoundary.csv and PCVparent*Boundary.csv, read
 * at ZebraflowWT.c:557-588): b_index [nx][ny][nz] is set to -1 and then to each
 * row's Bindex at its point; D, U, V, W are read and not kept, as the
 * reference does.  (The reference then marks and extrudes the parent segment,
 * :583-600, which is not part of this library.) */
int zf_read_boundary_csv(const char* path, int nx, int ny, int nz, const double* origin, double dx,
                         int32_t* b_index, int64_t* n_rows);

/* Fluid snapshot "X,Y,Z,Bindex,U,V,W,D,Bx,By,Bz,EulNeigh,Windex" (OUTPUT(),
 * ZebraflowWT.c:356-370): one row per listed point in DOMLIST order.  D..W,
 * eulneigh [n_listed] and bodyforce [3][n_listed] are in DOMLIST order;
 * windex is [nx][ny][nz]; eulneigh / windex NULL print 0. */
int zf_write_fluid_csv(const char* path, int nx, int ny, int nz, const double* origin, double dx,
                       const int32_t* b_index, const float* D, const float* U, const float* V, const float* W,
                       const float* bodyforce, const int32_t* eulneigh, const int32_t* windex);

/* Reads a fluid snapshot back (the reference's restart, :2649-2700): for each
 * row of a listed point of b_index, D, U, V, W, BODYFORCE and EulNeigh of
 * that point (DOMLIST order) and W_index ([nx][ny][nz]).  NULL outputs skip. */
int zf_read_fluid_csv(const char* path, int nx, int ny, int nz, const double* origin, double dx,
                      const int32_t* b_index, float* D, float* U, float* V, float* W, float* bodyforce,
                      int32_t* eulneigh, int32_t* windex, int64_t* n_rows);

/* Populations f [19][n] = feq(D, (U, V, W)), as the reference initialises F
 * from the restored moments (ZebraflowWT.c:2561-2570, :5253-5295); upload
 * them with zf_upload_populations. */
int zf_equilibrium_populations(int64_t n, const float* D, const float* U, const float* V, const float* W,
                               float* f);

/* Membrane snapshot, 21 columns (OUTPUT(), ZebraflowWT.c:429-442): rows of
 * every cell with status > -5000.  cell_id [n_cells] (the reference's 1-based
 * cell slot; NULL: c + 1), status [n_cells], x / vel [3][n_cells][n_node]
 * fp64, wall_tri / area_ratio / out_flag [n_cells][n_node], wrep / ftot /
 * fvol [3][n_cells][n_node], regress [n_cells].  NULL arrays print 0. */
int zf_write_membrane_csv(const char* path, int n_cells, int n_node, const int32_t* cell_id,
                          const int32_t* status, const double* x, const double* vel, const int32_t* wall_tri,
                          const float* wrep, const int32_t* regress, const float* area_ratio, const float* ftot,
                          const float* fvol, const int32_t* out_flag);

/* Nucleus snapshot, 13 columns (OUTPUT(), ZebraflowWT.c:446-459); layouts as
 * the membrane's with n_node_n nodes; neigh / neigh_flag [n_cells][n_node_n]. */
int zf_write_nucleus_csv(const char* path, int n_cells, int n_node_n, const int32_t* cell_id,
                         const int32_t* status, const double* xn, const double* vel_n, const float* ftot_n,
                         const int32_t* neigh, const int32_t* neigh_flag);

/* Nucleus spring snapshot "X,Y,Z,Cell,LX,LY,LZ,Stretch" (ZebraflowWT.c:461-504):
 * per nucleus edge its midpoint, n1 - n2 and |n1 - n2| 1e-6 / LMAX_N.
 * edge_n [n_edge_n][2] 1-based, lmax_n [n_edge_n] (zf_get_edge_params). */
int zf_write_nucleus_edges_csv(const char* path, int n_cells, int n_node_n, int n_edge_n, const int32_t* cell_id,
                               const int32_t* status, const double* xn, const int32_t* edge_n, const float* lmax_n);

/* Appends the cells' rows to VolumeAreaHistory.dat (ZebraflowWT.c:345-350;
 * the header is written when iter is 0).  cell_f [n_cells][8] as
 * zf_get_cell_geometry returns it (area, volume, centroid). */
int zf_append_volume_area(const char* path, int64_t iter, int n_cells, const int32_t* cell_id,
                          const int32_t* status, const float* cell_f, const int32_t* regress);

/* Reads a membrane (nucleus = 0, 21 columns) or nucleus (nucleus = 1, 13
 * columns) snapshot: the reference's cell restart (ZebraflowWT.c:5323-5420,
 * :5549-5574), n_node rows per cell.  With x NULL only *n_cells is returned;
 * otherwise cell_id, status [cap_cells] and x, vel, ftot [3][n_cells][n_node]
 * (NULL skips) are filled. */
int zf_read_cells_csv(const char* path, int nucleus, int n_node, int cap_cells, int* n_cells, int32_t* cell_id,
                      int32_t* status, double* x, double* vel, float* ftot);

/* Mesh files as the reference ships them (read at ZebraflowWT.c:1601-1922):
 * kind 0 "POINTS n ..." then n x 3 coordinates, kind 1 "CELLS n m" then n x 3
 * node ids (as stored, 1-based), kind 2 "LINES n m" then n x 2 node ids.
 * With values NULL only *n is returned. */
int zf_read_mesh_dat(const char* path, int kind, int* n, double* values, int cap);

/* Wall mesh files (read at ZebraflowWT.c:3724-3897): "POINTS n float" with the
 * coordinates, "POLYGONS n 4n" with "3 a b c" 0-based rows, and "CELL_DATA n"
 * / "NORMALS ..." with one normal per triangle.  Outputs as zf_set_wall takes
 * them: xyz [3][n], tri [3][m] 1-based (+1 as the reference adds), normals
 * [3][m].  With NULL outputs only the sizes are returned. */
int zf_read_wall_mesh(const char* nodes_path, const char* cells_path, const char* normals_path, int* n_node_w,
                      int* n_tri_w, float* xyz, int32_t* tri, float* normals, int cap_node, int cap_tri);

/* Legacy-VTK wall file of the post-processor (PostProWSSandPressure.c:375-433):
 * points, triangles, PRESSURE, WSSx/y/z and Valid per wall node (zf_wss). */
int zf_write_wall_vtk(const char* path, int n_node_w, const float* xyz, int n_tri_w, const int32_t* tri,
                      const float* pressure, const float* wss, const int32_t* valid);

#ifdef __cplusplus
}
#endif
#endif /* ZF_H */
