/*
 * alpineem_b200.h -- C ABI of the B200 FDTD solver library
 * (libalpineem_b200.so).
 *
 * The reference (DanRich123/AlpineEM) exposes its FDTD core as one
 * executable: master.py writes a positional input deck and runs
 * `./<solver> inputs.txt` (main_fdtd/master.py:438-441); the solver reads the
 * deck named by argv[1] (main_fdtd/fdtd_solver.f90:726-727), runs the time
 * loop (:4440-8299) and writes <name>.dat, <name>_geometry.bin and optional
 * <name>_video_*.bin next to the deck (:2355-2357, :8538-8807), which
 * utility_scripts/post_processor.py parses.  These entry points split that
 * executable into create / run / write so a caller (the FDTD-B200 launcher,
 * Python through ctypes) can drive it step by step.  Plain C types only.
 *
 * Errors: every function returns 0 on success and a negative AEM_ERR_* code
 * otherwise; aem_last_error() returns the message (for invalid decks, the
 * reference's own "ERROR: ..." text).  A handle is not thread-safe; distinct
 * handles are independent.  Device memory belongs to the handle and is freed
 * by aem_destroy.
 */
#ifndef ALPINEEM_B200_H
#define ALPINEEM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct aem_handle aem_handle;

#define AEM_OK 0
#define AEM_ERR_INPUT (-1)    /* invalid deck or missing side file (reference STOP "ERROR: ...") */
#define AEM_ERR_CUDA (-2)     /* CUDA runtime failure (no device, out of memory, launch error) */
#define AEM_ERR_ARG (-3)      /* bad argument to this API */
#define AEM_ERR_STATE (-4)    /* call out of order (e.g. write before the last step) */
#define AEM_ERR_DIVERGED (-5) /* the fields hold a non-finite value (extension `watchdog K`, checked every K steps) */

/* Deck grammar selector: the reference builds two solvers from one source
 * (fdtd_solver.f90:5-7); AEM_KMAX selects the constant-k periodic one. */
#define AEM_STANDARD 0
#define AEM_KMAX 1

/* Library version, encoded as major*10000 + minor*100 + patch. */
int aem_version(void);

/* Replaces the solver executable's start-up (fdtd_solver.f90:726-4355):
 * parse the deck at `inputs_path` (side files resolve against its
 * directory), build the model and upload it to the current CUDA device.
 * Output files go to `outdir` (NULL: the current directory, like the
 * reference).  Writes <name>_geometry.bin as the reference does. */
int aem_create_from_file(const char* inputs_path, int mode, const char* outdir, aem_handle** out);

/* Same as aem_create_from_file with the inputs in caller memory (copied
 * in): `deck_text` is the inputs.txt text (fdtd_solver.f90:726-1298
 * grammar); `ext_text` (may be NULL) holds extension lines, one "key value"
 * per line, as in the optional "<inputs>.b200" sidecar:
 *   pml_cells N      CPML thickness in cells (reference: 10, :1305-1318)
 *   geometry_bin no  skip building and writing <name>_geometry.bin
 *   cpml_grading m sigma_factor kappa_max alpha_max
 *                    CPML profile of order m with sigma_max =
 *                    sigma_factor (m+1) / (eta0 d) (reference: its fixed
 *                    profile, :1685-1706, :3404-3577)
 *   tfsf_inset N     TF/SF planes at index N and X-N (reference: npml+3,
 *                    :1386-1397)
 *   probe i j k      cell-centred Ex, Ey, Ez at cell (i, j, k) every step,
 *                    written to <name>_probes.dat (repeatable, at most 64)
 *   dft_freqs f0 f1 n   on-the-fly spectra (see aem_read_spectrum)
 *   watchdog K       check the fields for non-finite values every K steps
 *   autotune N       tune the general update's launch shape at the first
 *                    step, N steps per candidate (see aem_autotune)
 *   coef_precision 64   material (Ga, Gb, Drude Ja, Jb) and CPML (b, c,
 *                    kappa, den) tables evaluated on the GPU in FP64 and
 *                    rounded once (reference: FP32, :2832-2918, :3404-3666)
 * `bulk` replaces the bulk geometry file the deck names (:2051-2055):
 * bulk_count float32 material ids, x fastest, (nx, ny, nz) cells; NULL/0
 * when the deck has none.  Side files (gridded feeds) and outputs resolve
 * against `outdir`.  The reference reads these inputs from disk only. */
int aem_create_from_memory(const char* deck_text, const char* ext_text, const float* bulk, size_t bulk_count,
                           int mode, const char* outdir, aem_handle** out);

/* Parse and validate a deck (and extension lines) without a GPU, returning
 * the reference grid sizes X, Y, Z (fdtd_solver.f90:1316-1318).  Fails with
 * AEM_ERR_INPUT and the reference's "ERROR: ..." text where the reference
 * stops (:726-1298). */
int aem_check_deck(const char* deck_text, const char* ext_text, int mode, int sizes[3]);

/* Advance `nsteps` time steps of the reference loop (fdtd_solver.f90:4440,
 * one `counter` per step), never past the deck's step count. */
int aem_run(aem_handle* h, int nsteps);

/* aem_run with CUDA-graph replay: `steps_per_graph` steps are captured once
 * and replayed for every whole chunk (the kernels read the step number from
 * device memory).  Results equal aem_run's.  Steps before the first chunk
 * (the run's first step, far-field batch alignment) and the remainder run as
 * aem_run does.  The fused path needs an even chunk, far-field batching a
 * multiple of its 32-step batch.  No reference counterpart: the reference
 * launches every loop body from the host (fdtd_solver.f90:4440-8299). */
int aem_run_graph(aem_handle* h, int nsteps, int steps_per_graph);

/* Launch-shape autotuner of the general (two-kernel) H/E update: each of
 * 8 candidate shapes (z planes per CTA 4..64, rows per CTA 4 or 8) runs
 * the next `steps_per_candidate` steps of the run itself, timed with CUDA
 * events; the fastest shape of each kernel is kept.  Every cell's
 * arithmetic is the same under every shape, so the fields are those of an
 * untuned run.  shape (may be NULL) receives z planes H, rows H, z planes
 * E, rows E.  The fused path has no shape to tune (shape gets the unused
 * defaults).  The sidecar extension `autotune N` does this at the first
 * step.  No reference counterpart: the reference's OpenACC regions take the
 * compiler's launch shapes (fdtd_solver.f90:4443 and the like). */
int aem_autotune(aem_handle* h, int steps_per_candidate, int shape[4]);

/* Advance `count` independent runs (distinct handles on the same device,
 * each on its own stream) by `nsteps` each, replaying their graphs
 * round-robin so that small grids overlap on the GPU.  Each run's results
 * equal aem_run's.  This is the batched-instance driver that replaces the
 * reference's process-level fan-out (utility_scripts/parallel_kmax.py). */
int aem_run_batch(aem_handle* const* handles, int count, int nsteps, int steps_per_graph);

/* Raw per-step samples of the steps run so far, before the normalisation
 * that aem_write_outputs applies: kind 5 = voltage of port `index`
 * (Voltage_out, fdtd_solver.f90:8241-8243), kind 1 / 2 = reflected /
 * transmitted plane sums (:7005-7103; TE for kmax), kind 3 / 4 = their
 * kmax TM sums (:7105-7190), kind 6 = point probe (extension `probe i j k`;
 * index 3 p + c for probe p and component c = Ex, Ey, Ez, each the
 * cell-centred average of the phase-centre sample, :8273-8275).  Steps
 * first_step .. first_step+n-1 (1-based); im may be NULL.  Synchronises the
 * handle's stream. */
int aem_read_probe(aem_handle* h, int kind, int index, int first_step, int n, double* re, double* im);

/* On-the-fly spectrum of a per-step series (the run's sidecar extension
 * `dft_freqs f_start f_stop count`): X(f) = sum over the steps run so far of
 * x[m] exp(-i 2 pi f m dt), m = step - 1, dt the time step, accumulated in
 * FP64 with Kahan compensation by the per-step tap kernel.  kind / index as
 * aem_read_probe (1 / 2 reflected / transmitted plane sums, TE for kmax;
 * 3 / 4 their TM sums (kmax); 5 port `index`), on the raw samples.  Copies
 * min(n, count) values; freqs (Hz) and im may be NULL.  Returns the number
 * copied, or a negative error code.  Synchronises the handle's stream.
 * Replaces the post-hoc FFT of utility_scripts/post_processor*.py for these
 * series. */
int aem_read_spectrum(aem_handle* h, int kind, int index, int n, double* freqs, double* re, double* im);

/* Checkpoint / resume (no reference counterpart: the reference restarts a
 * run from step 1).  aem_checkpoint_save writes the whole run state after
 * the steps done so far to a file: every device buffer the handle set up
 * (fields, CPML psi, port lines, far-field bins and difference buffer,
 * per-step taps and spectra, tables) and the step counters.
 * aem_checkpoint_load restores it into a handle created from the same deck
 * (and extensions), at any step count; the run then continues as if it had
 * never stopped (fields bit-identical to an uninterrupted run).  A file from
 * another deck is rejected with AEM_ERR_ARG.  Not available while the
 * full-field export is on.  Both synchronise the handle's stream. */
int aem_checkpoint_save(aem_handle* h, const char* path);
int aem_checkpoint_load(aem_handle* h, const char* path);

/* The run's time step del_t in seconds (fdtd_solver.f90:1312, FP32
 * value widened). */
int aem_time_step(aem_handle* h, double* dt);

/* Phases of a time step, for per-phase device timing. */
#define AEM_NPHASE 8
#define AEM_PHASE_UPDATE_H 0     /* H update with sheets, TF/SF, CPML, PBC */
#define AEM_PHASE_UPDATE_E 1     /* E update with sheets, Drude, TF/SF, CPML, PBC */
#define AEM_PHASE_PORTS 2        /* lumped-port half-steps */
#define AEM_PHASE_FF_CURRENTS 3  /* Huygens-surface currents */
#define AEM_PHASE_FF_BIN 4       /* retarded-time binning */
#define AEM_PHASE_TAPS 5         /* plane sums, phase-centre, video */
#define AEM_PHASE_YEE 6          /* fused H+E update (decks without TF/SF, sheets, Drude, kmax) */
#define AEM_PHASE_OTHER 7

/* Per-phase timing (an extension; the reference prints only a total):
 * with profiling on, each kernel launch is bracketed by CUDA events on the
 * handle's stream.  aem_profile(h, 1) clears the record;
 * aem_profile_read returns milliseconds and launches per phase since. */
int aem_profile(aem_handle* h, int enable);
int aem_profile_read(aem_handle* h, double ms[AEM_NPHASE], long long launches[AEM_NPHASE]);

/* Kernels launched by the handle so far. */
int aem_launch_count(aem_handle* h, long long* n);

/* The far-field binning runs once per 32 steps over the buffered surface
 * currents (same sums as the reference's per-step binning,
 * fdtd_solver.f90:7643-7925); aem_flush bins the steps still buffered.
 * aem_write_outputs and the last step of the deck flush by themselves. */
int aem_flush(aem_handle* h);

/* The CUDA stream (cudaStream_t) the handle launches on, so callers can
 * order their own work and events after it. */
int aem_stream(aem_handle* h, void** stream);

/* Bytes copied host->device (model upload) and device->host (outputs,
 * probes, fields) by the handle so far. */
int aem_transfer_bytes(aem_handle* h, long long* h2d, long long* d2h);

/* Cells updated per step, (X-1)(Y-1)(Z-1) as the reference counts them
 * (fdtd_solver.f90:8315-8316), and the algorithmic HBM bytes one step must
 * move: 12 field values read + written and 1 material byte per cell, plus
 * 8 CPML psi values per cell of each CPML slab. */
int aem_workload(aem_handle* h, long long* cells, double* bytes_per_step);

/* Far-field work of one step: Huygens-surface cells (both planes of every
 * non-periodic axis, fdtd_solver.f90:7512-7641) and far-field angles; each
 * step bins face_cells x angles contributions (:7643-7925). */
int aem_far_field_size(aem_handle* h, long long* face_cells, int* angles);

/* Spectrum of a time series at arbitrary frequencies, on the GPU:
 *   out[2k] + i out[2k+1] = sum_{m<n} x[m] exp(-i 2 pi freqs[k] m dt).
 * x (n floats), freqs (nf doubles, Hz) and out (2*nf doubles) are device
 * pointers; the work is queued on `stream` (a cudaStream_t, NULL for the
 * default stream) and the call returns without waiting.  Replaces the
 * numpy FFT of the zero-padded series in utility_scripts/post_processor.py
 * (:160-215), whose bin k is this sum at k/((padding+1) n dt).  Accumulates
 * in FP64 in a fixed order (deterministic); takes a temporary device buffer
 * of 16 * chunks * nf bytes (chunks <= 64) from the stream-ordered pool. */
int aem_dft(const float* x, long long n, double dt, const double* freqs, int nf, double* out, void* stream);

/* Spectra of nseries series at once (every far-field angle and port of a
 * run): out[2*(s*nf + k)] + i out[2*(s*nf + k) + 1] =
 * sum_{m<n} x[s*ld + m] exp(-i 2 pi freqs[k] m dt).  FP64 samples (the
 * post-processor reads the .dat text as float64), FP64 accumulation;
 * device pointers, deterministic.  The spectra of post_processor.py
 * (:160-215, numpy's FFT of the zero-padded series, kept in the trusted
 * band :299-307) are these sums at the band's FFT bins. */
int aem_dft_batch(const double* x, long long ld, int nseries, long long n, double dt, const double* freqs, int nf,
                  double* out, void* stream);

/* aem_dft for callers that cannot allocate device memory (an application
 * that keeps all GPU memory in its own arena, a plugin host that forbids
 * allocation in its callbacks, a real-time loop that must not block on an
 * allocator).  Same arguments and the same results, bit for bit; it calls
 * no allocator.  The chunk sums live in one static device array of 1 MiB,
 * present on every GPU that loads the library until the process exits,
 * which bounds nf to 65536 frequencies: larger nf fails with AEM_ERR_ARG.
 * The first call on each device looks up that array's device address (with
 * the device current) and keeps it for the life of the process; make that
 * first call before any stream capture, and do not call this entry point on
 * a device after cudaDeviceReset (the kept address may be stale).
 * All calls share the array: calls that may overlap on the GPU (different
 * streams, or different threads) race and must be serialised by the
 * caller.  This entry point has no counterpart in the reference. */
int aem_dft_static(const float* x, long long n, double dt, const double* freqs, int nf, double* out, void* stream);

/* Steps done so far and the deck's step count. */
int aem_steps(aem_handle* h, int* done, int* total);

/* Wait for the device work queued on the handle's stream. */
int aem_synchronize(aem_handle* h);

/* Post-loop processing and the reference's output files
 * (fdtd_solver.f90:8338-8807): <name>.dat and, when requested by the deck,
 * <name>_video_*.bin.  Requires all steps to be done. */
int aem_write_outputs(aem_handle* h);

/* Time series after aem_write_outputs, as the .dat file holds them:
 *   kind 0 incident, 1 reflected, 2 transmitted (TE for kmax),
 *   3 reflected TM, 4 transmitted TM (kmax), 5 port voltage (index = port
 *   0..), 6 far-field E_theta (index = angle), 7 far-field E_phi.
 * Copies min(n, steps) values; im may be NULL. */
int aem_get_series(aem_handle* h, int kind, int index, double* re, double* im, int n);

/* Final field component in the reference's array layout (first index
 * fastest): comp 0..5 = Ex, Ey, Ez, Hx, Hy, Hz with the extents of
 * fdtd_solver.f90:3908-3913.  comp 6 = each cell's material index as the
 * run uses it (0 = background, r = the deck's r-th volume material) over
 * cells 1..N-1 of each axis, a periodic axis' duplicated layer left out
 * (the extents of <name>_geometry.bin).  `dims` receives the extents;
 * re/im must hold dims[0]*dims[1]*dims[2] values (pass NULL first to query
 * dims).  im may be NULL. */
int aem_get_field(aem_handle* h, int comp, int dims[3], double* re, double* im);

/* Reference grid sizes X, Y, Z (cells per axis + 1 + periodic layer,
 * fdtd_solver.f90:1316-1318). */
int aem_grid(aem_handle* h, int sizes[3]);

/* Bytes of device memory held by the handle. */
int aem_device_bytes(aem_handle* h, size_t* bytes);

/* Message of the last failing call on this handle (or of the last failing
 * aem_create_* when h is NULL).  Valid until the next call. */
const char* aem_last_error(aem_handle* h);

/* Free the handle and its device memory. */
int aem_destroy(aem_handle* h);

/* ---- design gradients -------------------------------------------------
 * The reference optimises material values with two solver runs per
 * iteration and a spectral overlap of their fields
 * (optimization_scripts/adjoint_optimization/adjoint_optimization.py:55-134,
 * the `fdtd.py` runs and the F1..F4 overlap).  These entry points return the
 * exact gradient of the discrete time loop instead: a forward run of the
 * deck with per-cell eps_r (and optionally sigma) inside a design box, then
 * the transposed update backwards in time, recomputing each checkpoint
 * segment.  Figure of merit F = |D|^2, D = sum_n c^n exp(-i 2 pi f n dt)
 * over all steps n, c^n the probe E component after step n.
 * Supported decks: standard solver, no periodic axes, lumped-port source
 * (no plane wave), no sheets, Drude poles or gridded ports; the design box
 * and the probe keep out of the CPML slabs and off the ports. */
typedef struct aem_design aem_design;

/* Build the run from the deck at `inputs_path`; the design box is cells
 * lo..lo+n-1 (reference indices).  precision 4: FP32 state, the reference's
 * arithmetic; 8: FP64 state (finite-difference checks). */
int aem_design_create(const char* inputs_path, const char* outdir, const int lo[3], const int n[3], int precision,
                      aem_design** out);

/* Probe: E component comp (0 x, 1 y, 2 z) at reference edge (i, j, k) and the
 * DFT frequency in Hz. */
int aem_design_set_probe(aem_design* d, int comp, int i, int j, int k, double freq_hz);

/* Design values per cell, n0*n1*n2 float32, x fastest; host or device
 * pointers.  sigma NULL keeps the conductivity of the deck's materials. */
int aem_design_set_eps(aem_design* d, const float* eps, const float* sigma);

/* Forward run over the deck's steps.  checkpoint_every < 1: a plain run;
 * otherwise the state is kept every that many steps for
 * aem_design_gradient.  fom gets F, dft (may be NULL) gets D (re, im). */
int aem_design_forward(aem_design* d, int checkpoint_every, double* fom, double dft[2]);

/* scale * dF/d eps_r and scale * dF/d sigma per design cell (float32,
 * x fastest, host or device pointers, either may be NULL).  Needs a
 * checkpointed aem_design_forward since the last aem_design_set_eps. */
int aem_design_gradient(aem_design* d, float* grad_eps, float* grad_sigma, double scale);

/* Overlap check (adjoint_optimization.py:121-134): the reference forms its
 * gradient from the overlap, at one frequency, of the spectra of a forward
 * and an adjoint run.  With enable != 0, aem_design_gradient also
 * accumulates on every design edge the DFTs at the probe frequency of the
 * forward E and of the adjoint field (32 B per edge), and
 * aem_design_gradient_overlap returns the gradient estimated from those two
 * spectra alone, assuming the adjoint field is a tone at that frequency, in
 * aem_design_gradient's layout and scale.  Its distance from the exact
 * gradient measures how far that assumption holds. */
int aem_design_set_overlap(aem_design* d, int enable);
int aem_design_gradient_overlap(aem_design* d, float* grad_eps, float* grad_sigma, double scale);

/* Device time in ms of the last forward [0] and gradient [1] calls, and the
 * kernels each launched. */
int aem_design_timing(aem_design* d, double ms[2], long long launches[2]);

/* Current field component comp (0..5 = Ex, Ey, Ez, Hx, Hy, Hz) of the run's
 * forward state in the reference layout (as aem_get_field); dims gets its
 * extents, out holds dims[0]*dims[1]*dims[2] values (NULL: dims only). */
int aem_design_get_field(aem_design* d, int comp, int dims[3], double* out);

/* The CUDA stream of the run (cudaStream_t). */
int aem_design_stream(aem_design* d, void** stream);

/* Message of the last failing call on d (of the last aem_design_create when
 * d is NULL). */
const char* aem_design_last_error(aem_design* d);

int aem_design_destroy(aem_design* d);

#ifdef __cplusplus
}
#endif

#endif /* ALPINEEM_B200_H */
