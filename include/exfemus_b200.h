/*
 * exfemus_b200.h -- C ABI of the B200 assembly + geometric-multigrid library.
 *
 * The library replaces the LASPACK backend of exFEMuS's MGSolBase/MGSolDA path:
 * element assembly (GenMatRhs), the level operators (ReadMatrix/ReadProl/ReadRest),
 * and the multigrid solve (MGSolve/MGStep with its smoothers and coarse solve) run on
 * one GPU.  Host code passes plain pointers and sizes; every call returns an EXF_*
 * status and never aborts.  A mesh owns the structured multilevel hierarchy; a system
 * (one per equation, like one MGSolBase object) owns its DOF map, boundary flags,
 * level matrices, transfer operators and vectors in device memory.  One CUDA stream
 * per system; a system is not thread-safe, independent systems are.
 *
 * Reference interfaces replaced (paths within danieleunibo/exfemus):
 *   include/MGSolverBase.h:118-361   MGSolBase (MGDofBcOp, GenMatRhs, MGSolve, MGStep)
 *   include/MGSolverDA.h             MGSolDA   (init_dof, GenBc, init, ReadProl, ReadRest)
 *   contrib/matrix/sparse_matrixM.h  SparseMatrixM / SparseMMatrixM handles
 *   contrib/matrix/numeric_vectorM.h:292-293  NumericVectorM::resid / matrix_mult
 *   contrib/matrix/linear_solverM.h:84-157    LinearSolverM::solve / adjoint_solve
 */
#ifndef EXFEMUS_B200_H
#define EXFEMUS_B200_H

#if defined(__GNUC__)
#define EXF_API __attribute__((visibility("default")))
#else
#define EXF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define EXF_OK 0
#define EXF_ERR_ARG 1           /* bad argument (null handle, size, level)          */
#define EXF_ERR_CUDA 2          /* CUDA runtime error (message in exf_last_error)   */
#define EXF_ERR_STATE 3         /* call order violated (e.g. solve before assembly) */
#define EXF_ERR_DIVERGED 4      /* NaN/Inf residual during the multigrid solve      */
#define EXF_ERR_NOT_CONVERGED 5 /* max_cycles reached above the tolerance           */
#define EXF_ERR_SINGULAR 6      /* zero pivot in the coarsest direct factorisation  */
#define EXF_ERR_NOMEM 7         /* device allocation failed                         */
#define EXF_ERR_UNSUPPORTED 8   /* option not implemented for this system or kernel */
#define EXF_ERR_IO 9            /* an output file could not be written              */

/* system kinds: MGSolT (one quadratic variable) and coupled MGSolNS (NS_EQUATIONS==1:
 * dim quadratic velocity components + one linear pressure) */
#define EXF_KIND_T 0
#define EXF_KIND_NS 1
/* the two variables of the turbulence template's coupled kappa-omega system
 * (MGSolTBK, template_appl/turb-ckw/SRC/MGSolverTBKW.C, TBK_EQUATIONS 5, Wilcox 2006 with
 * the low-Reynolds corrections): the system's matrix has no kappa-omega coupling blocks,
 * so each variable is one scalar system (quadratic, like MGSolT) that reads the other
 * through exf_sys_couple, the Navier-Stokes velocity likewise, and the element wall
 * distances of exf_sys_set_wall */
#define EXF_KIND_K 2
#define EXF_KIND_W 3
/* one direction of the fluid-structure template's mesh displacement (MGSolDS,
 * template_appl/fsi/SRC/MGSolverDS.C:321-700 with ALE_MOVING): one quadratic variable,
 * assembled from the FSI velocity and the old displacements of exf_sys_set_ds */
#define EXF_KIND_DS 4

/* boundary-condition presets: the per-node bc_read rules of the workloads */
#define EXF_BC_HEAT_DIRICHLET 1  /* T = 0 on every wall                              */
#define EXF_BC_CAVITY 2          /* no-slip, u = 1 on the lid interior, p gauge node 0 */
#define EXF_BC_CHANNEL 3         /* inlet x=0 prescribed, no-slip walls, natural outlet */
#define EXF_BC_BOUSS_NS 4        /* no-slip on all walls, p gauge node 0             */
#define EXF_BC_BOUSS_T 5         /* T prescribed on x=0 and x=1, adiabatic y walls   */

/* smoothers */
#define EXF_SMOOTH_GS 0          /* multi-colour Gauss-Seidel (scalar systems)      */
#define EXF_SMOOTH_VANKA 1       /* multi-colour pressure-node Vanka (NS)           */
#define EXF_SMOOTH_GMRES_ILU 2   /* GMRES(30) + ILU, the reference's default level    */
                                 /* solver (scalar systems, FP64 precision)          */

/* precision of the V-cycle */
#define EXF_PREC_FP64 0          /* everything FP64                                 */
#define EXF_PREC_MIXED 1         /* FP32 V-cycle inside FP64 defect correction      */

/* Vanka kernel selection (exf_mg_params.vanka_kernel): all compute the same update and
 * differ only in the order of floating-point sums.  AUTO uses BULK on 3D FP32 levels
 * with more than four waves of rows and ROWS elsewhere (each measured fastest there); BULK
 * and ROWS give the same bits. */
#define EXF_VANKA_AUTO 0
#define EXF_VANKA_TILE 1         /* one CTA per patch, iterate staged in shared memory */
#define EXF_VANKA_ROWS 2         /* star-row residual kernel + patch-solve kernel      */
#define EXF_VANKA_STREAM 3       /* ROWS with the 3D FP32 star rows copied to shared    */
                                 /* memory by cp.async (persistent warps)               */
#define EXF_VANKA_BULK 4         /* ROWS with the 3D FP32 star rows of each persistent  */
                                 /* CTA streamed by bulk copies through mbarrier stages */

typedef struct {
  int dim;          /* 2 (quad9/quad4) or 3 (hex27/hex8)                          */
  int nlev;         /* geometric levels                                            */
  int n0[3];        /* elements per direction on level 0                           */
  double box[6];    /* x0,x1,y0,y1,z0,z1                                           */
  int device;       /* CUDA device ordinal                                         */
} exf_mesh_desc;

typedef struct {
  double inv_re;    /* _IRe (viscosity); heat diffusivity = inv_prdl*inv_re        */
  double inv_prdl;  /* _IPrdl                                                      */
  double rho;       /* density factor                                              */
  double rhocp;     /* rho*cp                                                      */
  double inv_dt;    /* 1/dt of the mass term (0 = steady)                          */
  double penalty;   /* Dirichlet penalty scale: Ipenalty = det_side*penalty        */
  double upwind_ns; /* UP_WIND_NS                                                  */
  double upwind_t;  /* UP_WIND_T                                                   */
  double ifr;       /* _IFr                                                        */
  double dirg[3];   /* _dirg                                                       */
  double buoy;      /* Boussinesq source coefficient: f += buoy*T*dirg             */
  double traction;  /* 1: natural NS sides whose bc1 has bit 2 get the pressure    */
                    /* traction rhs -n_a p_old phi (the reference's MESHNUMBER 1) */
} exf_phys;

typedef struct {
  double eps;          /* stop when ||b-Ax||/||b|| <= eps                          */
  int max_cycles;
  int gamma;           /* cycles per coarse visit (1 = V)                          */
  int nu_pre, nu_post; /* smoothing sweeps                                         */
  int double_below_top;/* 1: sweeps doubled below the top level (MGStep)           */
  int smoother;        /* EXF_SMOOTH_*                                             */
  double omega;        /* Vanka damping                                            */
  double corr_damp;    /* coarse-correction factor (reference 0.95)                */
  int cond_corr;       /* 1: reference's conditional coarse correction: x += 0.95 P x_c */
                       /* only when the coarse accuracy is below the pre-smoothing one */
                       /* (src/MGSolverBase.C:262-263)                                 */
  int reverse_colours; /* 1: colours swept in reverse order                        */
  int precision;       /* EXF_PREC_*                                               */
  int use_graph;       /* 1: replay each V-cycle from a captured CUDA graph        */
  int vanka_kernel;    /* EXF_VANKA_*                                              */
  int stop_test;       /* EXF_STOP_*                                               */
  int fp32_blocks;     /* mixed precision: 1 = the Vanka sweeps read the FP32 velocity */
                       /* blocks (FP32 storage throughout the V-cycle) with the row    */
                       /* kernel; 0 = row-scaled FP16 block records (default)          */
  int coarse_iters;    /* 0: direct solve on level 0 (default); with the GMRES + ILU   */
                       /* smoother, n > 0 runs that level solver for n iterations there */
                       /* instead, as MGStep does (60, src/MGSolverBase.C:222)          */
} exf_mg_params;

/* stop tests of exf_mg_solve.  A level's accuracy is what the reference's level solver
 * reports (LASPACK's LastAcc): ||b - A x|| / ||b|| of the iterate before the last sweep of
 * a smoothing call (of the coarsest level: after its solve). */
#define EXF_STOP_RELRES 0     /* ||b - A x|| / ||b|| <= eps after a cycle                  */
#define EXF_STOP_REFERENCE 1  /* rest < eps*(1 + ||b||), rest = the top level's accuracy of */
                              /* the cycle's post-smoothing (src/MGSolverBase.C:201); in    */
                              /* mixed precision rest is the FP64 relative residual        */

typedef struct {
  int cycles;
  int converged;
  double rel_res;
  double bnorm;
  double seconds;      /* device time of the solve (CUDA events on the system stream) */
  double hist[256];    /* relative residual after each cycle                       */
  double last_acc;     /* the top level's accuracy of the last cycle (EXF_STOP_*)  */
} exf_solve_stats;

typedef struct exf_mesh exf_mesh;
typedef struct exf_sys exf_sys;

EXF_API const char *exf_last_error(void);
EXF_API const char *exf_version(void);

/* --- mesh: structured multilevel hierarchy (the restated gencase output) ------------
 * replaces MGMesh::read_c (src/MGMesh.C:493-908) for generated boxes */
EXF_API int exf_mesh_create(const exf_mesh_desc *desc, exf_mesh **out);
EXF_API int exf_mesh_destroy(exf_mesh *m);
/* --- mesh from host arrays: the hierarchy MGMesh::read_c holds (src/MGMesh.C:493-908)
 * after reading gencase's mesh file, one subdomain (the LASPACK path is single-process):
 *   nnodes[L]   _NoNodes[L]: Q2 nodes of level L.  Nodes are numbered level-nested as
 *               init_dof requires (src/MGSolverDA.C:880-951): the nodes of level L are the
 *               top nodes 0..nnodes[L]-1, so the Q1 (pressure) nodes of level L are the Q2
 *               nodes of level L-1, and those of level 0 are the first nvert0 nodes
 *   nvert0      _NoNodes of the linear coarse mesh: vertices of level 0
 *   xyz         _xyz, [dim][nnodes[nlev-1]] component-major
 *   nel[L]      _NoElements[0][L]
 *   conn        _el_map[0]: the volume elements of every level, level after level
 *               (_off_el[0]), [sum nel][9 | 27] top node numbers in libMesh Quad9/Hex27
 *               local order, vertices first
 *   neigh       _el_neighbor[0]: [sum nel][4 | 6] level-local index of the element across
 *               each side (libMesh side order), -1 on the boundary
 *   parent      [sum_{L>=1} nel[L]] level-local index of each element's parent on level
 *               L-1 (gencase's elem_sto parent, USER_APPL/gencase/src/MGGenCase.C:306-346);
 *               NULL when the transfer operators come from exf_sys_set_transfer instead
 * The children of an element must be the 2^dim sub-cells of its reference element with
 * the parent's orientation (uniform refinement); the library places each child by the
 * parent vertex it contains and checks that the prolongation reproduces the fine node
 * coordinates (EXF_ERR_ARG otherwise).  Smoother and assembly colourings are greedy
 * first-fit colourings taken in (z, y, x) coordinate order; on a structured box they
 * equal the colourings of exf_mesh_create, so both give the same bits. */
typedef struct {
  int dim;
  int nlev;
  int device;
  const int *nnodes;
  int nvert0;
  const double *xyz;
  const int *nel;
  const int *conn;
  const int *neigh;
  const int *parent;
} exf_mesh_data;
EXF_API int exf_mesh_upload(const exf_mesh_data *d, exf_mesh **out);
/* --- mesh by uniform refinement of a coarse quad9 / hex27 mesh (the role of gencase:
 * libMesh uniformly_refine(nlev - 1) and printMesh's level-nested numbering,
 * USER_APPL/gencase/src/MGGenCase.C:176-181, 234-...):
 *   nnode0, xyz0  the coarse mesh's Q2 nodes, [dim][nnode0] component-major; its nvert0
 *                 vertices are nodes 0..nvert0-1
 *   nel0, conn0   its elements, [nel0][9 | 27] in libMesh Quad9/Hex27 local order
 * Every element splits into the 2^dim sub-cells of its reference element with its own
 * orientation; new nodes take the element's triquadratic (biquadratic) map at their
 * reference coordinates, so curved elements stay curved, and points on shared edges and
 * faces are created once.  Level L+1 keeps the nodes of level L with their numbers and
 * appends its new ones; neighbours are matched by side vertices; the parent of child
 * e * 2^dim + c is e.  exf_mesh_refine_arrays returns the hierarchy as exf_mesh_upload
 * takes it (host arrays owned by the library, released by exf_mesh_data_free);
 * exf_mesh_refine uploads it, transfers from the parents. */
typedef struct {
  int dim;
  int nlev;
  int device;
  int nnode0;
  int nvert0;
  const double *xyz0;
  int nel0;
  const int *conn0;
} exf_mesh_coarse;
EXF_API int exf_mesh_refine_arrays(const exf_mesh_coarse *c, exf_mesh_data *out);
EXF_API void exf_mesh_data_free(exf_mesh_data *d);
EXF_API int exf_mesh_refine(const exf_mesh_coarse *c, exf_mesh **out);
EXF_API int exf_mesh_info(const exf_mesh *m, int lev, int *nnodes, int *nel, int *nvert0);
EXF_API int exf_mesh_get_xyz(const exf_mesh *m, double *xyz);               /* [dim][ntop]    */
EXF_API int exf_mesh_get_conn(const exf_mesh *m, int lev, int *conn, int *neigh, int *colour);

/* --- system: MGSolBase::MGDofBcOp (src/MGSolverBase.C:139-159) --------------------- */
EXF_API int exf_sys_create(exf_mesh *m, int kind, exf_sys **out);      /* init_dof + pattern   */
EXF_API int exf_sys_destroy(exf_sys *s);
EXF_API int exf_sys_ndof(const exf_sys *s, int lev, int *ndof);
EXF_API int exf_sys_get_node_dof(const exf_sys *s, int lev, int *node_dof);   /* _node_dof[L] */
EXF_API int exf_sys_bc_preset(exf_sys *s, int preset);                     /* GenBc            */
EXF_API int exf_sys_set_bc(exf_sys *s, const int *bc0, const int *bc1);
EXF_API int exf_sys_get_bc(const exf_sys *s, int *bc0, int *bc1);
EXF_API int exf_sys_nnz(const exf_sys *s, int lev, long *nnz);
EXF_API int exf_sys_get_pattern(exf_sys *s, int lev, int *rowptr, int *col); /* ReadMatrix    */
/* transfer operators; pass NULL arrays to query nnz only */
EXF_API int exf_sys_get_prol(exf_sys *s, int lev, long *nnz, int *rowptr, int *col, double *val);
EXF_API int exf_sys_get_rest(exf_sys *s, int lev, long *nnz, int *rowptr, int *col, double *val);
EXF_API int exf_sys_get_colours(exf_sys *s, int lev, int *ncolours, int *colour_of_item);
/* transfer operators from gencase's operator datasets (ReadProl src/MGSolverDA.C:2011-2230,
 * ReadRest :2236-2444; written by compute_prol_qq / compute_res_qq,
 * USER_APPL/gencase/src/MGGenCase.C:2308-2569; datasets DIM0<b>, LEN0<b>, POS0<b>, VAL0<b>
 * of the Prol<L-1>_<L> / Rest<L+1>_<L> files, contrib/matrix/sparse_MmatrixM.C:194-264):
 *   kind  0 = prolongation into level lev (rows: nodes of lev, columns: nodes of lev-1),
 *         1 = restriction into level lev (rows: nodes of lev, columns: nodes of lev+1)
 *   block 2 = the quadratic (Q2 node) block "22", 1 = the linear (Q1 node) block "11"
 *   dim   DIM0<b>: {rows, columns}; len LEN0<b>: rows+1 cumulative row offsets;
 *   pos   POS0<b>: level-local column nodes; val VAL0<b>: the entries
 * Every variable of the block uses the node operator, as in the reference.  Restriction rows
 * are scaled by bc0 % 2 of their top-level DOF when applied (:2423-2425), so the flags may
 * change later.  Columns are sorted per row; entries are kept as given. */
EXF_API int exf_sys_set_transfer(exf_sys *s, int lev, int kind, int block, const int dim[2], const int *len,
                                 const int *pos, const double *val);
/* the writer side of exf_sys_set_transfer: one block of a level's transfer operator in
 * gencase's dataset layout (what compute_prol_qq / compute_res_qq write,
 * USER_APPL/gencase/src/MGGenCase.C:2308-2569), for the caller to store as DIM0<b>, LEN0<b>,
 * POS0<b>, VAL0<b>; kind and block as for exf_sys_set_transfer.  dim receives {rows,
 * columns} and *nnz the entry count; len (rows + 1), pos and val (nnz each) are filled when
 * not NULL (a first call with NULL arrays sizes them).  Columns are sorted per row.
 * EXF_ERR_STATE when the block has not been built or supplied yet. */
EXF_API int exf_sys_get_transfer(exf_sys *s, int lev, int kind, int block, int dim[2], long *nnz, int *len, int *pos,
                                 double *val);
/* check a level's sparsity against gencase's matrix datasets (ReadMatrix,
 * src/MGSolverDA.C:1785-2009; LEN0<b>/POS0<b> of block b = 22 (Q2 rows, Q2 columns) or 21
 * (Q2 rows, Q1 columns)): EXF_OK when every row holds exactly the node columns the library
 * built from the elements (in any order, as LASPACK sorts them, operats.c:813),
 * EXF_ERR_ARG with the first differing row otherwise */
EXF_API int exf_sys_check_pattern(exf_sys *s, int lev, int block, const int dim[2], const int *len, const int *pos);
/* coupling: T reads the NS velocity, NS reads T for buoyancy (get_el_sol of the
 * other equation, src/MGSolverBase.C:336-354); a kappa / omega system reads the NS
 * velocity and the other turbulence variable; NS coupled to both kappa and omega
 * systems takes the eddy viscosity IRe (1 + mu_t) of the turbulence template
 * (template_appl/turb-ckw/SRC/MGSolverNS.C:256-293); a displacement system reads the
 * velocity of an NS system and, for dy / dz, the dx system's x_old.  The library keeps
 * a pointer to other: destroying other clears the coupling (the next assembly that
 * needs it returns EXF_ERR_STATE) */
EXF_API int exf_sys_couple(exf_sys *s, exf_sys *other);
/* kappa / omega systems: the wall distance of every element (_mgmesh._dist: level 0's
 * elements first, then level 1's, ...) and nu_wall = mu / rho of the omega wall value
 * 6 nu_wall / (BETASTAR y^2) */
EXF_API int exf_sys_set_wall(exf_sys *s, const double *dist, double nu_wall);
/* displacement systems (EXF_KIND_DS): the direction dir (0 = dx, 1 = dy, 2 = dz, the
 * reference's _dir), the time step dt, and the top-level node fields [dim][ntop] the
 * element matrices read: u_fsi, the FSI velocity, and d_old, the old displacement of every
 * direction.  Elements whose centre node has bc0 >= 2 are solid (displacement row
 * d = u_fsi dt + d_old of the direction), the rest fluid (100 dt times the Laplacian,
 * masked by bc0 % 2 and zero on interface nodes, bc0 > 3); a boundary side whose last
 * node has an even bc0 gets the penalty det_side / dt with the rhs
 * bc1 % 2 (u_fsi dt + d_old) of direction 0, as the reference writes it for every
 * direction (MGSolverDS.C:610-650) */
EXF_API int exf_sys_set_ds(exf_sys *s, int dir, double dt, const double *u_fsi, const double *d_old);
/* u_fsi = d_old = NULL: the fields stay on the device as the reference's _data_eq x_old
 * views: u_fsi the velocity components of the NS system coupled with exf_sys_couple
 * (x_old's first dim*ntop entries), d_old of direction dir the system's own x_old and of
 * direction 0 the dx system coupled with exf_sys_couple (itself when dir = 0) */
/* moving_mesh with FINE_MOVEMENT (MGSolverDS.C:724-744): at each exf_sys_xold_update
 * (and so in exf_timestep_loop) the mesh's node coordinates of direction dir move by
 * x - x_old on the device; every later assembly reads the moved mesh, and
 * exf_mesh_get_xyz, the output and exf_mesh_wall_dist the moved coordinates */
EXF_API int exf_sys_set_mesh_motion(exf_sys *s, int moving);
/* MGMesh::B_dist (src/MGMesh.C:1285-1350): for every element of every level (level 0's
 * first), the distance from its centre (mean of its nodes) to the nearest centre (mean of
 * the side's nodes) of a wall side of its level; a boundary side is a wall when all its
 * nodes have wall_node[n] != 0 (wall_node: [ntop], the reference's user predicate) */
EXF_API int exf_mesh_wall_dist(const exf_mesh *m, const int *wall_node, double *dist);

/* --- fields (host buffers) ---------------------------------------------------------- */
EXF_API int exf_sys_set_xold(exf_sys *s, const double *xold);   /* x_old[top]             */
EXF_API int exf_sys_get_xold(exf_sys *s, double *xold);
EXF_API int exf_sys_set_x(exf_sys *s, const double *x);         /* x[top]                 */
EXF_API int exf_sys_get_x(exf_sys *s, double *x);
EXF_API int exf_sys_xold_update(exf_sys *s);                    /* x_old[top] = x[top]    */
EXF_API int exf_sys_set_source(exf_sys *s, const double *qe);   /* per top-level element  */
EXF_API int exf_sys_set_rhs(exf_sys *s, const double *b);
EXF_API int exf_sys_get_rhs(exf_sys *s, double *b);

/* --- assembly: GenMatRhs (MGSolverNS.C:108-717, MGSolverT.C:93-525) ----------------- */
EXF_API int exf_gen_mat_rhs(exf_sys *s, const exf_phys *ph, int lev, int mode);
/* every level, top mode 1, others mode 0: the same matrices and rhs, bit for bit, as
 * exf_gen_mat_rhs level by level, in one launch per element colour for all levels */
EXF_API int exf_assemble_all(exf_sys *s, const exf_phys *ph);
EXF_API int exf_get_matrix(exf_sys *s, int lev, double *val);   /* values in pattern order  */
EXF_API int exf_set_matrix(exf_sys *s, int lev, const double *val);

/* --- solve: MGSolve / MGStep (src/MGSolverBase.C:163-289) on device state ------------- */
EXF_API int exf_mg_solve(exf_sys *s, const exf_mg_params *p, exf_solve_stats *st);
/* the time / Picard loop of MGEquationsSystem::eqnmap_timestep_loop
 * (src/MGEquationsSystem.C:422-432): nsteps times, for each of the nsys systems in order,
 * its MGTimeStep (MGSolverNS.C:722-750, MGSolverT.C:530-561): assemble every level with
 * phys[k], solve with params[k], x_old = x.  Coupled systems see each other's x_old as
 * updated within the step.  Per (step, system) the cycles and device seconds of the solve
 * go to cycles[step*nsys + k] and seconds[...] when those are not NULL.  A solve that ends
 * at its cycle limit above its tolerance does not stop the loop (MGSolve does not stop
 * MGTimeStep): every step runs, and the loop then returns EXF_ERR_NOT_CONVERGED; any
 * other failure stops the loop and returns its status. */
EXF_API int exf_timestep_loop(exf_sys *const *sys, int nsys, const exf_phys *phys, const exf_mg_params *params,
                              int nsteps, int *cycles, double *seconds);

/* --- solution output (MGEquationsSystem::print_soln, src/MGEquationsSystem.C:606-721,
 * with MGMesh::print_conn_lin_hf5 / print_xmf_topology / print_xmf_geometry,
 * src/MGMesh.C:439-477, 1074-1195, and MGSolDA::print_u / print_xml_attrib,
 * src/MGSolverDA.C:1184-1290).  HDF5 is replaced by raw little-endian binary files that the
 * XDMF file addresses by byte offset (Format="Binary", Seek), one file per HDF5 file of the
 * reference, datasets in the reference's order:
 *   <dir>/<basemesh><connlin>.bin       MSH0CONN: int32 [nel * 2^dim][4 | 8], each Q2
 *                                       element as its 2^dim linear sub-cells
 *   <dir>/<basemesh>.<step>.bin         X1, X2, X3: float64 [nnodes] each (X3 = 0 in 2D)
 *   <dir>/<basesol>.<step>.bin          one float64 [nnodes] dataset per variable
 *   <dir>/<basesol>.<step>.xmf          Grid "Mesh": Time, Topology (Quadrilateral |
 *                                       Hexahedron), Geometry X_Y_Z, one node Attribute
 *                                       per variable
 * <step> is t_step zero-padded to ndigits.  Quadratic variables are written at every node;
 * linear ones (pressure) are read at the element vertices and interpolated to the other
 * nodes with the element's linear basis, as print_u does. */
typedef struct {
  const char *dir;       /* _inout_dir: directory of every file ("" or NULL: current)  */
  const char *basesol;   /* BASESOL: stem of the solution files, e.g. "sol"            */
  const char *basemesh;  /* BASEMESH: stem of the mesh files, e.g. "mesh"              */
  const char *connlin;   /* CONNLIN: suffix of the sub-cell connectivity, "_conn_lin"  */
  int ndigits;           /* digits of the step number in file names (1..9)             */
  int t_step;            /* step number (>= 0)                                         */
  double time;           /* <Time Value> (the reference writes t_step * dt)            */
} exf_soln_out;
/* one top-level mesh with node fields, for exf_write_xdmf (host arrays only) */
typedef struct {
  int dim;               /* 2 (quad9) or 3 (hex27)                                      */
  int nnodes;
  const double *xyz;     /* [dim][nnodes] component-major                              */
  int nel;
  const int *conn;       /* [nel][9 | 27] libMesh local order, vertices first          */
  int nvars;
  const char *const *names;  /* [nvars] dataset and attribute names                    */
  const int *order;      /* [nvars] 2: quadratic (every node), 1: linear (vertices)    */
  const double *vals;    /* [nvars][nnodes]; a linear variable is read at vertices only */
} exf_node_fields;
EXF_API int exf_write_xdmf(const exf_node_fields *f, const exf_soln_out *o);
/* print_soln of nsys systems on one mesh: every variable of every system in order
 * (MGSolNS: u, v[, w], p; MGSolT: T unless names are given), each scaled by
 * refvalue[var] (NULL: 1), from x of the top level. */
EXF_API int exf_print_soln(exf_sys *const *sys, int nsys, const char *const *names, const double *refvalue,
                           const exf_soln_out *o);
/* MGEquationsSystem::print_case (src/MGEquationsSystem.C:814-935): the initial state
 * (x_old) of every variable with its boundary flags <name>bd (bc1) and <name>vl (bc0)
 * (MGSolDA::print_bc, src/MGSolverDA.C:1418-1520), three node attributes per variable, in
 * <dir>/<basesol>.<step>.xmf/.bin (basesol as BASECASE) over the base mesh coordinates
 * <basemesh>.bin, without <Time>; exf_write_xdmf_case writes given node fields so */
EXF_API int exf_print_case(exf_sys *const *sys, int nsys, const char *const *names, const double *refvalue,
                           const exf_soln_out *o);
EXF_API int exf_write_xdmf_case(const exf_node_fields *f, const exf_soln_out *o);
/* unit-level operations on host buffers (NumericVectorM::resid / matrix_mult);
 * exf_resid with b == NULL returns r = A x */
EXF_API int exf_resid(exf_sys *s, int lev, const double *x, const double *b, double *r);
EXF_API int exf_restrict(exf_sys *s, int lev, const double *r_fine, double *b_coarse); /* lev = coarse */
EXF_API int exf_prolong(exf_sys *s, int lev, const double *x_coarse, double *y_fine);  /* lev = fine   */
EXF_API int exf_smooth(exf_sys *s, int lev, const exf_mg_params *p, int nsweeps, double *x, const double *b);
EXF_API int exf_coarse_solve(exf_sys *s, const double *b, double *x);
/* y = ILUPrecond(c) of level lev (LASPACK's ILU(0) of the level matrix, factored once per
 * assembly; contrib/laspack/precond.c:75-110, factor.c:25-320), y may be c; scalar systems */
EXF_API int exf_ilu_apply(exf_sys *s, int lev, const double *c, double *y);
EXF_API int exf_sys_transpose(exf_sys *s);                      /* A[L] <- A[L]^T, all levels */

/* --- discrete adjoint of the T solve (LinearSolverM::adjoint_solve semantics) ------------
 * forward: assemble all levels with the current x_old/sources and solve A T = b.
 * backward: solve A^T lambda = dJ/dT on the transposed hierarchy (colours reversed) and
 * return dJ/dq_e (per top element) and dJ/dg (per top DOF: derivative with respect to
 * the Dirichlet data value held in x_old at Dirichlet DOFs). */
EXF_API int exf_adjoint_forward(exf_sys *s, const exf_phys *ph, const exf_mg_params *p, exf_solve_stats *st);
EXF_API int exf_adjoint_backward(exf_sys *s, const exf_phys *ph, const exf_mg_params *p, const double *djdx,
                         double *djdq, double *djdg, exf_solve_stats *st);

#define EXF_FMA_CHAINS 8
#define EXF_FMA_ITERS 4096

/* --- timing of one kernel class on device-resident data (CUDA events) -----------------
 * what: 0 = SpMV residual, 1 = smoother sweep, 2 = assembly (all levels), 3 = V-cycle,
 * 4 = factorisation of the coarsest level (as each solve after an assembly pays it),
 * 5 = FP64 FMA throughput probe: 4 CTAs of 256 threads per SM, each thread running
 *     EXF_FMA_CHAINS independent chains of EXF_FMA_ITERS fma (2 flops each);
 * 6 = bounded-wait probe: one kernel waits, with a short limit, on a barrier phase that
 *     nothing completes; returns EXF_ERR_CUDA with the run-out message, the status every
 *     bounded in-kernel wait (the BULK smoother's stage barriers) reports, and leaves the
 *     context usable;
 * 7 = ILU factorisation of level lev (scalar systems; the GMRES + ILU level solver pays it
 *     once per assembly), 8 = one ILUPrecond application on level lev (in place on r);
 * avg_ms = average duration per launch group over reps, precision per exf_mg_params */
EXF_API int exf_time_op(exf_sys *s, int what, int lev, const exf_mg_params *p, const exf_phys *ph, int reps,
                double *avg_ms);
EXF_API int exf_sync(exf_sys *s);
/* device-side timing marks on the system stream (8 slots) and the number of kernels the
 * library has launched so far (all systems) */
EXF_API int exf_event_record(exf_sys *s, int slot);
EXF_API int exf_event_elapsed(exf_sys *s, int slot_a, int slot_b, double *ms);
EXF_API long long exf_launch_count(void);
/* Allocation-free residual: r = b - A x on level lev and ||r||^2, for callers that cannot
 * allocate device memory while they run (the host application owns every allocation,
 * or memory is reserved before a run).  x, b, r and norm2 are DEVICE buffers owned by the
 * caller (ndof doubles; norm2 one double).  The norm's per-block partial sums live in a
 * fixed file-scope device array of EXF_STATIC_PARTIALS doubles held by every GPU that
 * loads the library; levels needing more partial sums are rejected with EXF_ERR_ARG.
 * Nothing is allocated or freed.  The first call on a device resolves the array's device
 * address, so make that first call before any stream capture.  The call returns once the
 * system stream has finished it (it synchronizes that stream); while that stream is being
 * captured it returns EXF_ERR_STATE and leaves the capture alone.  All calls share the
 * array: calls that overlap on the GPU race.  It has no counterpart in the reference. */
#define EXF_STATIC_PARTIALS 32768
EXF_API int exf_resid_norm_static(exf_sys *s, int lev, const double *x, const double *b, double *r,
                                  double *norm2);
/* algorithmic bytes of one residual (spmv: every matrix row once, FP32 or FP64 values)
 * and of one smoother sweep on level lev (GS: every row once; Vanka: every star row of
 * every patch in the value format the sweep reads, since each colour recomputes the
 * residuals of its stars from the iterate at its start) */
EXF_API int exf_level_bytes(exf_sys *s, int lev, int precision, double *spmv_bytes, double *sweep_bytes);

#ifdef __cplusplus
}
#endif
#endif
