/*
 * cupyram_b200.h - C ABI of the B200 split-step Pade parabolic-equation engine.
 *
 * The engine replaces the range march of clapeyre/cupyram (CuPyRAM.run):
 * profile interpolation, range-index updates, Galerkin assembly, the np
 * Pade tridiagonal sweeps per range step, the self-starter and the
 * receiver / TL-grid extraction.  Everything here is plain C: host pointers,
 * sizes and int status codes; no CUDA or torch types cross the boundary, so
 * ctypes, cffi or any C FFI can bind it.
 *
 * Units: metres, seconds, Hz, m/s, g/cm^3, dB/wavelength.  Complex numbers are
 * stored as interleaved (re, im) float64 pairs.
 *
 * Threading: one engine per host thread.  Each engine owns a CUDA stream on
 * the device that was current when it was created.  The library never calls
 * exit() or abort(); every failure is reported by a status code and the text
 * from cr_last_error().
 */
#ifndef CUPYRAM_B200_H
#define CUPYRAM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CR_ABI_VERSION 3
/* Largest number of Pade terms a ray may use. */
#define CR_MAX_NP 10

/* Status codes returned by every entry point. */
enum cr_status {
    CR_OK = 0,
    CR_EINVAL = 1,    /* invalid argument or inconsistent batch description */
    CR_ECUDA = 2,     /* CUDA runtime error (text in cr_last_error)          */
    CR_EPADE = 3,     /* Pade root finding did not converge                   */
    CR_ETIMEOUT = 4,  /* a device-side wait gave up: the batched march's
                         waits for its bulk copies are bounded (flag bit 1)  */
    CR_ENAN = 5,      /* a ray produced a non-finite field (see cr_ray_flags) */
    CR_ENOMEM = 6,    /* device or host allocation failed                     */
    CR_ESTATE = 7     /* call made in the wrong order (e.g. march before upload) */
};

/* Arithmetic form of the range march. */
enum cr_precision {
    CR_PLAIN_C128 = 0,   /* complex128 field and sweeps, FP64 arithmetic          */
    CR_CHOSEN_C64R = 1,  /* complex64 factors, workspace and sweeps (FP32 arithmetic);
                            the Pade terms are combined in FP64 and the field is
                            kept in complex128                                    */
    CR_CHOSEN_C64 = 2,   /* complex64 factors and workspace with an FP32 inner loop:
                            sweeps, couplings, M u and the term combination in
                            FP32; the factorisation and the stored field stay
                            FP64 / complex128                                     */
    CR_C64_REFINED = 3   /* CR_CHOSEN_C64R plus one iterative-refinement step per
                            Pade term and range step: the residual
                            M u - (M + pd2 D) x of the complex64 solve in FP64,
                            its correction solved with the same complex64
                            factors and added.  Rays on the column kernel or
                            in the product form run complex128 instead       */
};

/*
 * One ray (one "calculation" of the reference: an environment at one
 * frequency).  The grid and step sizes are per ray; the reference's shared
 * grid is the special case where all rays carry the same values.
 * Mirrors the per-calculation state of CuPyRAM.setup (cupyram/cupyram.py:528-726).
 */
typedef struct cr_ray {
    double freq;         /* Hz                                                  */
    double c0;           /* reference sound speed (m/s); k0 = 2*pi*freq/c0      */
    double zs, zr;       /* source / receiver depth (m)                         */
    double dz, dr;       /* depth and range step (m)                            */
    double zmax;         /* bottom of the computational grid incl. the layer (m) */
    double lyrw_lambda;  /* absorbing-layer width in metres (lyrw * lambda)     */
    double attnf;        /* attenuation at the bottom of the layer (dB/wavelength, 10 in RAM) */
    double rs;           /* range beyond which the stability constraints are dropped (m) */
    int32_t nz;          /* interior depth points; the grid has nz+2 rows       */
    int32_t nr;          /* march steps after the self-starter                  */
    int32_t np;          /* Pade terms, 1..CR_MAX_NP                            */
    int32_t ns;          /* stability constraints 0..2                          */
    int32_t ndr, ndz;    /* output decimation in range / depth                  */
    int32_t nvr, nvz;    /* output ranges / output depths (TL grid rows)        */
    int32_t env;         /* index into the environment table                    */
    int32_t reserved;
    int64_t line_off;    /* element offset of this ray's TL line in tll / cpl   */
    int64_t grid_off;    /* element offset of this ray's [nvz][nvr] grid, or -1 */
} cr_ray;

/*
 * One environment record.  Its arrays live contiguously in the float64 pool
 * starting at `off`, in this order:
 *   z_ss[n_zss], rp_ss[n_rss], cw[n_rss][n_zss],
 *   z_sb[n_zsb] (absolute depths), rp_sb[n_rsb],
 *   cb[n_rsb][n_zsb], rhob[n_rsb][n_zsb], attn[n_rsb][n_zsb],
 *   rb[n_bt], zb[n_bt]   (bathymetry ranges and depths, extended to rmax)
 * Profiles are stored profile-major (one contiguous depth profile per update
 * range), the transpose of the reference's cw[depth, range] input.
 */
typedef struct cr_env {
    int32_t n_zss, n_rss, n_zsb, n_rsb, n_bt, reserved;
    int64_t off;
} cr_env;

typedef struct cr_batch {
    int32_t n_rays, n_envs;
    const cr_ray* rays;
    const cr_env* envs;
    const double* pool;
    int64_t pool_len;
    int32_t precision;      /* enum cr_precision                                */
    int32_t compute_grids;  /* 0: TL line only; 1: also TL / CP grids           */
    int64_t line_len;       /* total elements of tll (and of cpl, complex)      */
    int64_t grid_len;       /* total elements of tlg (and of cpg, complex)      */
} cr_batch;

/* Caller-owned host output buffers (cpl, cpg interleaved complex). */
typedef struct cr_outputs {
    double* tll;   /* [line_len]                  TL line (dB)          */
    double* cpl;   /* [2*line_len]                complex pressure line */
    double* tlg;   /* [grid_len] or NULL          TL grid (dB)          */
    double* cpg;   /* [2*grid_len] or NULL        complex pressure grid */
} cr_outputs;

/* Timing and work counters of the last march (device clock). */
typedef struct cr_stats {
    double march_ms;          /* self-starter + range march, CUDA events        */
    double assemble_ms;       /* initial profile assembly                       */
    double h2d_ms, d2h_ms;    /* last upload / download                         */
    double point_updates;     /* sum over rays of nz * nr                       */
    int64_t h2d_bytes, d2h_bytes;
    int32_t kernel_launches;  /* kernels launched by the last cr_march           */
    int32_t rays_failed;      /* rays whose field went non-finite               */
    int32_t tile_rays;        /* rays per tile in the device layout             */
    int32_t n_tiles;
    int64_t device_bytes;     /* device memory held by the engine               */
    int32_t column_rays;      /* rays marched by the column-parallel kernel      */
    int32_t column_launches;  /* cluster launches of the last cr_march           */
    int32_t queue_ctas;       /* CTAs of the persistent batched launch (0: none,
                                 or one launch per lanes-per-ray value)        */
    int32_t precision_used;   /* enum cr_precision the march runs in: the
                                 batch's, except that a batch with a source in
                                 the first depth cell (zs < dz) runs the
                                 complex128 product form in every form         */
    double create_ms;         /* host wall time of cr_create                    */
    double pade_ms;           /* host wall time of the device Pade sets in it   */
    double tuner_row_step_s;  /* measured batched cost the column policy used:
                                 one row of one step of a tile alone (0: the
                                 policy was forced by CUPYRAM_B200_COL)         */
    double tuner_updates_per_s; /* measured batched throughput it used          */
    double tuner_slots;       /* batched tiles the device holds at once         */
} cr_stats;

typedef struct cr_engine cr_engine;

/* ABI version of the loaded library (CR_ABI_VERSION). */
int cr_abi_version(void);

/*
 * Pade coefficients of exp(i*k0*dr*(sqrt(1+X)-1)) (ip=1) or of the
 * self-starter operator (ip=2), product form, FP64.
 * Replaces cupyram/pade.py:180-273 compute_pade_coefficients(freq, c0,
 * np_pade, ns, dr, ip).  pd1, pd2: 2*np doubles each (re, im interleaved).
 * Returns CR_EPADE when Laguerre iteration fails to converge
 * (cupyram/pade.py:146-147 raises ValueError there).
 */
int cr_pade(double freq, double c0, int np, int ns, double dr, int ip,
            double* pd1, double* pd2);

/*
 * Pade coefficients of n independent (freq, c0, np, ns, dr, ip) jobs, solved
 * on the current CUDA device, one thread per job, by the same FP64
 * construction as cr_pade.  Replaces the host loops that call
 * compute_pade_coefficients once per environment and frequency
 * (cupyram/cupyram.py:706-726, :984-999, :1040-1060) and the unused
 * cupyram/pade.py:276-317 compute_pade_coefficients_batch.
 *   freq, c0, dr: [n] doubles; np, ns, ip: [n] int32 (np 1..CR_MAX_NP,
 *   ns 0..2, ip 1 or 2).  Host memory.
 *   pd1, pd2: [n][CR_MAX_NP] complex (2*CR_MAX_NP doubles per job,
 *   interleaved; zeros past the job's np).  status: [n] int32, CR_OK,
 *   CR_EPADE (Laguerre did not converge) or CR_EINVAL per job.
 * Returns CR_OK when every job succeeded, else the first failing job's code
 * (its index in cr_global_error); CR_EINVAL for bad arguments, CR_ECUDA /
 * CR_ENOMEM for device failures.  Synchronous; uses temporary device memory.
 */
int cr_pade_batch(int n, const double* freq, const double* c0, const int32_t* np,
                  const int32_t* ns, const double* dr, const int32_t* ip,
                  double* pd1, double* pd2, int32_t* status);

/*
 * Build an engine for a batch: validates the description, computes the Pade
 * sets of every ray (self-starter, march, march without stability
 * constraints) on the device in FP64 (as cr_pade_batch), sorts rays into device tiles by work and
 * allocates device memory.  Replaces the set-up half of CuPyRAM.run
 * (cupyram/cupyram.py:528-726: setup, profl, Pade batch).
 */
int cr_create(const cr_batch* batch, cr_engine** out);

/* Copy the batch's environments and per-ray parameters to the device. */
int cr_upload(cr_engine* e);

/*
 * Self-starter + full range march on the device, inputs already resident.
 * Replaces the loop of CuPyRAM.run (cupyram/cupyram.py:296-317: updat,
 * _propagate_step, _outpt) and CuPyRAM.selfs (:1001-1063).  Synchronous.
 */
int cr_march(cr_engine* e);

/* Copy outputs to the caller's host buffers (layout given by line_off/grid_off). */
int cr_download(cr_engine* e, const cr_outputs* out);

/* cr_upload + cr_march + cr_download: the whole CuPyRAM.run on the device. */
int cr_run(cr_engine* e, const cr_outputs* out);

/* Cell-averaged transmission loss, computed on the device from the last
 * march's TL-grid outputs (no counterpart in the reference, whose grid can
 * only be downloaded whole): cell (j, c) of a ray averages |p|^2 over the sz
 * x sr grid outputs at rows j*sz .. j*sz+sz-1 and output ranges c*sr ..
 * c*sr+sr-1, p^2 = |cp|^2 / r, and reports -10 log10 of the mean.
 * tl_cells: host buffer of n_rays * ncz * ncr floats, [ray][j][c]; cells
 * beyond a ray's grid are NaN.  Needs batch->compute_grids. */
int cr_cell_tl(cr_engine* e, int sz, int sr, int ncz, int ncr, float* tl_cells);

/* Override one ray's Pade set: which = 0 self-starter (1-X)^-2 factor,
 * 1 self-starter ip=2, 2 march, 3 march after rs.  n terms (<= CR_MAX_NP). */
int cr_set_pade(cr_engine* e, int ray, int which, int n, const double* pd1, const double* pd2);

/* Per-ray status flags of the last march (bit 0: non-finite field; bit 1: a
   bounded wait for the batched march's bulk copies gave up, CR_ETIMEOUT). */
int cr_ray_flags(cr_engine* e, int32_t* flags, int n);

int cr_get_stats(const cr_engine* e, cr_stats* st);

/* Copy the last error message (NUL-terminated, truncated to len). */
int cr_last_error(const cr_engine* e, char* buf, size_t len);

/* Message of the last failure of a call that had no engine (cr_create, cr_pade). */
int cr_global_error(char* buf, size_t len);

void cr_destroy(cr_engine* e);

/*
 * The cost rule the engine's column policy applies at cr_create, on the host:
 * is_column[i] = 1 when ray i's lockstep march in a batched tile,
 * (nz + 2)(nr + 4 + 4 x operator changes) x row, exceeds 1.25 x the whole
 * batch's balanced time, sum(nz nr) / updates_per_s.  row is the larger of
 * row_step_s (a tile alone) and in_flight / updates_per_s, in_flight being
 * the batch's rays, at most slots x the mean rays per tile (slots <= 0: no
 * cap).  cr_create takes the costs from the engine's tuner (measured once per
 * device and precision form; cr_stats.tuner_*), and sends a chosen ray to the
 * column kernel when its column also fits a cluster.  No counterpart in the
 * reference, which sizes one grid for all rays (cupyram/cupyram.py:596-597).
 */
int cr_plan_columns(const cr_batch* batch, double row_step_s, double updates_per_s, double slots,
                    int32_t* is_column);

/*
 * Engines take their device memory from a stream-ordered pool per device that
 * keeps freed memory for the next engine, so that creating an engine per
 * batch (as CuPyRAM.run() does for every call) costs no fresh cudaMalloc /
 * cudaFree after the first.  CuPy's default memory pool plays this part for
 * the reference; cr_release_cache returns the pooled memory that no live
 * engine holds to the device, as cupyram/benchmark.py:35-36 does with
 * get_default_memory_pool().free_all_blocks().
 */
int cr_release_cache(void);

/*
 * Size in bytes of the device scratch built into the library for
 * cr_march_static (a file-scope device array; every GPU that loads the
 * library holds it until the process exits).
 */
#define CR_STATIC_SCRATCH_BYTES (32u * 1024u * 1024u)

/*
 * cr_march_static - the whole march without allocating anything.
 *
 * No counterpart in the reference: CuPyRAM allocates its device arrays with
 * CuPy for every run.  This entry point is for callers that cannot allocate
 * device memory at the moment they want a march: a real-time sonar or
 * tactical-decision loop that forbids allocation after start-up (an
 * allocation can take unbounded time and may synchronise the device), or a
 * plug-in running inside a host application whose device memory is owned by
 * that application's own pool, where an extra cudaMalloc fails or fragments
 * the pool.  The caller owns the outputs; the per-ray tables, Pade
 * coefficients (computed on the device), environments and the march
 * workspace live in the library's CR_STATIC_SCRATCH_BYTES of device scratch.
 *
 *   batch    host description, as for cr_create (rays, envs and pool in host
 *            memory).  Limit: the batch's scratch need (per-ray tables, the
 *            pool, and 68 bytes per row per ray of march workspace, rows
 *            counted as the batch's deepest nz + 2 for every ray) must not
 *            exceed CR_STATIC_SCRATCH_BYTES; otherwise CR_EINVAL with the
 *            required size in cr_global_error.
 *   dev_out  DEVICE pointers: tll [line_len] doubles and cpl [line_len]
 *            complex (interleaved); tlg / cpg [grid_len] when
 *            batch->compute_grids is set.  Same ragged layout as cr_download.
 *   stream   cudaStream_t as void* (NULL: the legacy default stream).
 *
 * Returns after the march has finished on `stream`.  Calls no cudaMalloc,
 * cudaFree or other allocating routine; on success it takes no host heap
 * memory either (a failure stores its message for cr_global_error).
 * The first call on a device does a one-time set-up with that device
 * current: it looks up the scratch array's device address
 * (cudaGetSymbolAddress), and the driver loads the library's kernels and
 * their fixed local memory.  Make that first call during the caller's own
 * initialisation, before any stream capture.  The address is kept with the
 * handle of the context it was looked up in; a call in a new context of the
 * device (after cudaDeviceReset, say) repeats the look-up, so no call uses an
 * address of a context that no longer exists.  Every call shares the one scratch array and
 * it keeps the last call's contents (everything a march needs is rewritten
 * or cleared by the call itself), so calls whose work overlaps on the GPU -
 * from two threads, or on two streams of one device - race and must be
 * serialised by the caller.  Only the plain complex128 form is supported.
 */
int cr_march_static(const cr_batch* batch, const cr_outputs* dev_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUPYRAM_B200_H */
