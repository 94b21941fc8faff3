/*
 * cs_b200.h -- entry points of libcsgpu.so beyond the reference ABI.
 *
 * The reference GPU backend (src/cuda.cu) has no counterpart for these: they
 * expose the device-resident path (spectrum already in HBM, enqueue without a
 * host round trip), session introspection, and the dedispersion kernel.  The
 * reference-compatible ABI is in coherent_search.h.
 */
#ifndef CS_B200_H
#define CS_B200_H

#include <stddef.h>
#include <stdint.h>
#include "coherent_search.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int ntiles;          /* 128-trial tiles (never straddling a chunk) */
    long long nchunks;   /* reference chunk table entries */
    int nslot;           /* base profile + decimations */
    int npad;            /* tensor-core N (profile columns, padded) */
    int kpad;            /* tensor-core K (2*nharms, padded) */
    int smem_bytes;      /* dynamic shared memory per CTA */
    int grid;            /* persistent CTAs launched */
    long long total;     /* trials */
    unsigned rec_capacity;
    int kernel;          /* 0: generic fused kernel, 1: warp-specialised
                            kernel for the default ladder (nharms 60, 32,
                            16), 2: the FP64 search (--precision f64),
                            3: the column-tile kernel with TMA-staged
                            windows (default ladder, hidr 0.5) */
} CsB200Info;

int cs_b200_session_info(const GpuSession *s, CsB200Info *info);

/* One persistent launch over the tiles of several spectra (no counterpart
 * in the reference, which searches one file per call): sessions ss[0..n-1],
 * all FP32 and of one warp-specialised configuration (the same nharms and
 * decimation ladder at m 16), each with its own geometry, tables and record
 * buffer.  d_amps[i] is session i's device spectrum (NULL array or entry:
 * its own buffer).  Each session's spectrum maximum, then one kernel whose
 * CTAs walk a single list of (spectrum, tile) work items, are queued on
 * `stream` (NULL: the first session's stream) after the work already queued
 * on every session's stream; every session's stream then waits for the
 * launch, so cs_b200_session_collect on each session returns its
 * candidates, the same as those of its own search.  Calls on one device are
 * serialised.  Returns 0, or -1 with a message. */
int cs_b200_multi_enqueue(GpuSession **ss, int n, const float *const *d_amps,
                          double threshold, void *stream);

/* The same multi-spectrum search recorded once as a CUDA graph and replayed
 * (no counterpart in the reference; its list driver makes one search call
 * per file, src/cli.c:976-1099, src/search.c:1292-1341).  create captures,
 * on a private stream, what cs_b200_multi_enqueue queues: each spectrum's
 * counter clears and maximum, the argument-table copy into constant memory
 * (from pinned memory the graph owns) and the persistent launch.  launch
 * replays it on `stream` (NULL: the first session's stream) after the work
 * queued on every session's stream, and every session's stream then waits
 * for it, so cs_b200_session_collect returns each session's candidates --
 * equal to those of cs_b200_multi_enqueue on the same spectra.  The graph
 * holds the sessions' buffer and spectrum addresses: launch returns -2 when
 * a session was reloaded or grew its record buffer since the capture (an
 * overflow that collect reported), and the graph must be freed before any of
 * its sessions.  Replays on one device are serialised like
 * cs_b200_multi_enqueue.  create returns NULL with a message on error;
 * launch returns 0, -2, or -1 with a message. */
typedef struct CsMultiGraph CsMultiGraph;
CsMultiGraph *cs_b200_multi_graph_create(GpuSession **ss, int n, const float *const *d_amps,
                                         double threshold);
int cs_b200_multi_graph_launch(CsMultiGraph *g, void *stream);
void cs_b200_multi_graph_free(CsMultiGraph *g);

/* Device address of the session's spectrum buffer (namps float2). */
float *cs_b200_session_device_amps(GpuSession *s);

/* Enqueue one search of a device-resident spectrum (NULL: the session's own
 * buffer) on the session stream without synchronising.  A non-NULL `stream`
 * (a cudaStream_t) is the spectrum's producer: the search starts after the
 * work queued on it so far.  The kernel is bracketed by CUDA events;
 * cs_b200_session_collect reports its time. */
int cs_b200_session_enqueue_device(GpuSession *s, const float *d_amps,
                                   double threshold, void *stream);

/* Wait for the enqueued search, read back and order the candidates exactly
 * as cs_gpu_session_run does.  Returns 0, 1 if the record buffer overflowed
 * (it has been grown; enqueue again), or -1 on error. */
int cs_b200_session_collect(GpuSession *s, double threshold, CandidateList *out,
                            float *kernel_ms);

int cs_b200_session_sync(GpuSession *s);

/* Like cs_b200_session_collect, but the records never leave the device: they
 * are harvested, ordered and collapsed there exactly as search_file's
 * post-processing does (src/search.c:1467-1478: remove_duplicates with
 * dr_tol when `remove`, else a stable frequency sort; then remove_harmonics
 * with numharm / harm_tol when `harm_remove`), and only the resulting list
 * comes back.  Returns 0, 1 if the record buffer overflowed (grown; enqueue
 * again), or -1. */
int cs_b200_session_collect_collapsed(GpuSession *s, double threshold, int remove,
                                      double dr_tol, int harm_remove, int numharm,
                                      double harm_tol, CandidateList *out, float *kernel_ms);

/* The two halves of cs_b200_session_collect_collapsed.  _enqueue waits for
 * the search (it reads the record count), then queues the collapse on the
 * session stream and returns 0, 1 (record buffer grown: enqueue the search
 * again) or -1; _wait synchronises and hands over the list.  Between the
 * two the caller can queue work for other sessions. */
int cs_b200_session_collapse_enqueue(GpuSession *s, double threshold, int remove,
                                     double dr_tol, int harm_remove, int numharm,
                                     double harm_tol);
int cs_b200_session_collapse_wait(GpuSession *s, CandidateList *out, float *kernel_ms);

/* ---- batched search of many spectra -------------------------------------
 * No reference counterpart: the reference searches one file per call
 * (src/search.c:1388-1406) and rebuilds its GPU session whenever the file
 * length changes.  Here requests (one spectrum each, any length and search
 * parameters) run on a pool of `nslots` slots, each a session with its own
 * host thread and CUDA stream.  One request's table building and upload
 * overlap another's kernel, and a slot's device buffers are reused across
 * lengths.  A slot takes a request only while the device memory that all
 * slots hold stays within `mem_budget` bytes (0: no limit); idle slots give
 * their buffers back when another slot needs the room. */
typedef struct CsBatch CsBatch;

CsBatch *cs_gpu_batch_create(int device, int nslots, size_t mem_budget);

/* Queue the search of one spectrum over [lofreq, hifreq] Hz (lobin != 100
 * overrides the low edge, blocksize 0 means 65536), as search_file would run
 * it.  ft and *p are copied; ft->amps (host memory; pinned memory uploads at
 * full speed) must stay valid until the request is waited for.  Returns the
 * request id, or -1. */
long long cs_gpu_batch_submit(CsBatch *b, const FFTFile *ft, const SearchParams *p,
                              double lofreq, double hifreq, int lobin, int blocksize,
                              double threshold);

/* Wait for one request.  *out receives its raw candidates exactly as
 * cs_gpu_session_run returns them (owned by the caller); queued_ms and run_ms
 * (optional) the time it waited for a slot and the time the slot spent on
 * it.  Returns 0, -1 (unknown id, or the search failed) or -2 (cancelled). */
int cs_gpu_batch_wait(CsBatch *b, long long id, CandidateList *out, double *queued_ms,
                      double *run_ms);

/* Load every slot for the geometry of a request (ft->N, ft->namps, ft->T and
 * the band; ft->amps is not read) and return once all slots have built their
 * tables and grown their device buffers to it.  A server calls it before
 * traffic with its largest request: a slot that grows while serving frees
 * device memory, and cudaFree waits for the whole device, other slots'
 * searches included.  Returns 0, or -1 if a slot failed. */
int cs_gpu_batch_warm(CsBatch *b, const FFTFile *ft, const SearchParams *p, double lofreq,
                      double hifreq, int lobin, int blocksize);

/* Cancel a request that no slot has taken yet: it is dropped from the
 * queue and its wait returns -2 with an empty list.  Returns 0 when
 * cancelled, 1 when it is already on a slot or finished (it completes as
 * usual), -1 for an unknown id.  The request still has to be waited for. */
int cs_gpu_batch_cancel(CsBatch *b, long long id);

/* Device bytes the slots hold now (the figure admission holds to the
 * budget), or -1. */
long long cs_gpu_batch_device_bytes(CsBatch *b);

/* Requests submitted and not yet waited for. */
int cs_gpu_batch_pending(CsBatch *b);

/* Finishes the queued requests, then frees everything (results not waited
 * for are dropped). */
void cs_gpu_batch_free(CsBatch *b);

/* ---- time series -> normalised spectrum ---------------------------------
 * The in-memory `realfft + rednoise` of src/datpipe.c:101-253: forward real
 * FFT packed PRESTO-style (bin 0 = DC, Nyquist), then the running block-median
 * normalisation (defaults startwidth 6, endwidth 100, endfreq 6 Hz,
 * src/cli.c).  Output: N/2 complex bins (interleaved floats), the layout of
 * FFTFile.amps and of a session's device spectrum.  One run at a time per
 * plan.  NULL / -1 where the reference's rednoise stops with an error. */
typedef struct CsSpectrum CsSpectrum;

CsSpectrum *cs_spectrum_create(long long N, double dt, int startwidth, int endwidth,
                               double endfreq, int device);

/* Device buffers: d_series N floats, d_amps N floats (N/2 complex); on
 * `stream` (a cudaStream_t; NULL: the plan's stream). */
int cs_spectrum_run_device(CsSpectrum *s, const float *d_series, float *d_amps, void *stream);

/* Host buffers; copies in and out and waits. */
int cs_spectrum_run(CsSpectrum *s, const float *h_series, float *h_amps);

void cs_spectrum_free(CsSpectrum *s);

/* ---- duty cycles on the device ------------------------------------------
 * measure_ducy (src/candidate.c:305-329) for candidates of a spectrum that is
 * already in device memory (a session's buffer, cs_b200_session_device_amps):
 * the m = 64 FP64 profile of each candidate's harmonics, its boxcar widths
 * for the search's fsp / maxfrac, and width / bins of the best one.
 * ducy_out[i] is NaN where measure_ducy leaves it NaN (nharm < 1, r <= 0;
 * also nharm > 64).  Returns 0, or -1 on error. */
typedef struct CsDucy CsDucy;
CsDucy *cs_ducy_create(double fsp, double maxfrac, int device);
int cs_ducy_run_device(CsDucy *d, const float *d_amps, long long namps, long long N,
                       const Candidate *cands, long long ncand, double *ducy_out,
                       void *stream);
void cs_ducy_free(CsDucy *d);

/* ---- prepsubband's time-domain clipping -------------------------------
 * How many spectra PRESTO's clip_times (third_party/presto/src/clipping.c)
 * would replace when the reference's front end runs with -clip clip_sigma
 * (its default, 6) on the 8-bit filterbank at d_raw ([nspec][nchan], SIGPROC
 * order): every full block of L spectra, running statistics carried from
 * block to block.  d_flags (device, nspec / L * L bytes, may be NULL) gets 1
 * for each such spectrum.  The unclipped dedispersion equals the clipped
 * run exactly when *nclipped is 0 (counted over every full block, also ones
 * a run with a shorter numout never reads); otherwise cs_clip_levels gives
 * what cs_dedisp_run_device_clipped substitutes.
 * d_scratch: device memory of cs_clip_scratch_bytes(nspec, L) bytes, 256-byte
 * aligned, kept by the caller across calls; NULL makes the call allocate and
 * free its own, which synchronises the device and can take far longer than
 * the work.  Returns 0 or -1. */
size_t cs_clip_scratch_bytes(long long nspec, int L);
int cs_clip_count(const uint8_t *d_raw, long long nspec, int nchan, int L, float clip_sigma,
                  long long *nclipped, uint8_t *d_flags, void *d_scratch, size_t scratch_bytes,
                  void *stream, int device);

/* cs_clip_count plus the channel levels clip_times leaves after each block
 * (its good_chan_levels, clipping.c:118-160), which it writes over the
 * spectra it replaces: d_levels (device, [nspec / L][nchan] floats, SIGPROC
 * channel order like d_raw).  d_flags and d_levels are required; with
 * clip_sigma <= 0 nothing is written.  Returns 0 or -1. */
int cs_clip_levels(const uint8_t *d_raw, long long nspec, int nchan, int L, float clip_sigma,
                   long long *nclipped, uint8_t *d_flags, float *d_levels, void *d_scratch,
                   size_t scratch_bytes, void *stream, int device);

/* ---- SIGPROC filterbank header (in libcoherent_search.so) --------------
 * The header read_filterbank_header parses (third_party/presto/
 * src/sigproc_fb.c:240-345) and the band edges PRESTO derives from it
 * (:435-441): lofreq = fch1 - (nchans - 1) * |foff| (the centre of the lowest
 * channel), chanwid = |foff|.  header_bytes is where the [nspectra][nchans]
 * 8-bit samples start.  Returns 0, or -1 (message on stderr) for a file the
 * device front end cannot take (not 8-bit unsigned, several IFs, ascending
 * channels). */
typedef struct {
    int nchans, nbits, nifs, ibeam, telescope_id, machine_id, signedints;
    double tstart, tsamp, fch1, foff, src_raj, src_dej;
    char source_name[80], rawdatafile[80];
    long long header_bytes, nspectra;
    double lofreq, chanwid;
} CsSigproc;
int cs_sigproc_read_header(const char *path, CsSigproc *h);

/* The value prepsubband pads every DM series with: PRESTO's running mean
 * (update_stats) of DM 0's n output samples.  In libcoherent_search.so. */
double cs_prep_pad_value(const float *x, long long n);

/* ---- subband dedispersion of 8-bit filterbank data ---------------------
 * The prepsubband stage of the reference's raw-data front end
 * (src/prep_dedisp.c:444-466 tables, :1104-1275 block driver; PRESTO
 * dispersion.c dedisp_subbands :218-267 and float_dedisp :322-365; the
 * reference GPU kernels third_party/presto/src/cuda.cu:557-597, 704-768).
 * Input: raw spectra [nspec][nchan] of unsigned 8-bit samples in SIGPROC
 * order (highest frequency first), as the file holds them.  Output: for DM
 * d, out[d * out_stride + t], t < the returned length, bit-identical to the
 * reference's FP32 result for the same delays (cs_dedisp_run_device_clipped
 * adds prepsubband's -clip; no masking, downsampling or barycentring). */
typedef struct CsDedisp CsDedisp;

/* Delay tables as prep_dedisp.c computes them for DMs lodm + i*dmstep:
 * idispdt[nchan] (channel delays in samples, ascending frequency),
 * offsets[ndm*nsub] (subband offsets per DM), blocks per read and the
 * subbanding DM.  lofreq: centre of the lowest channel (MHz); chanwid > 0. */
int cs_dedisp_tables(int nchan, int nsub, int ndm, double lodm, double dmstep, double lofreq,
                     double chanwid, double dt, int spectra_per_subint, int *idispdt,
                     int *offsets, int *blocks_per_read, double *avgdm);

/* Plan for up to max_spectra input spectra; NULL on invalid geometry (a
 * delay outside the reference's limits, or sums that would not be exact). */
CsDedisp *cs_dedisp_create(int nchan, int nsub, int ndm, const int *idispdt, const int *offsets,
                           int spectra_per_subint, int blocks_per_read, long long max_spectra,
                           int device);

/* Output points per DM the reference writes for nspec spectra, at most
 * numout (numout < 0: no cap). */
long long cs_dedisp_output_length(const CsDedisp *d, long long nspec, long long numout);

/* Device buffers: d_out 16-byte aligned, out_stride a multiple of 4.
 * Enqueued on `stream` (a cudaStream_t, NULL for the plan's stream). */
int cs_dedisp_run_device(CsDedisp *d, const uint8_t *d_raw, long long nspec, long long numout,
                         float *d_out, long long out_stride, void *stream,
                         long long *nout_written);

/* The run prepsubband makes with -clip (its default): the spectra d_flags
 * marks (cs_clip_levels) take their block's channel levels d_levels, and the
 * subband and DM sums are evaluated in FP32 in the reference's order
 * (channels, then subbands, ascending; dispersion.c:245-264, 346-362).  With
 * no spectrum flagged it equals cs_dedisp_run_device bit for bit.  The first
 * clipped run allocates the plan's float subbands (nsub x the plan's stride
 * floats).  Returns 0 or -1. */
int cs_dedisp_run_device_clipped(CsDedisp *d, const uint8_t *d_raw, long long nspec,
                                 long long numout, const uint8_t *d_flags, const float *d_levels,
                                 float *d_out, long long out_stride, void *stream,
                                 long long *nout_written);

/* Host buffers; copies in and out and waits.  -1 also when a bounded wait
 * inside the DM stage gave up (the output is then not valid). */
int cs_dedisp_run(CsDedisp *d, const uint8_t *h_raw, long long nspec, long long numout,
                  float *h_out, long long out_stride, long long *nout_written);

/* CUDA-event times of the last run's subband and DM kernels (ms); waits for
 * the run and returns -1 when one of its DM-stage waits gave up. */
int cs_dedisp_last_times(CsDedisp *d, float *subband_ms, float *dm_ms);

void cs_dedisp_free(CsDedisp *d);

/* ---- session reuse ---------------------------------------------------
 * cs_gpu_session_free keeps up to CS_B200_SESSION_PARK freed sessions per
 * process (default 2; 0 frees at once, as the reference does) and the next
 * cs_gpu_session_create on the same device reloads one for its geometry,
 * instead of making and freeing its device and pinned buffers per file (the
 * reference's drivers free and recreate the session whenever the spectrum
 * length changes, src/search.c:1388-1406).  Results are the same bits.  A
 * parked session still holds its device memory; this frees every parked
 * session and returns how many there were. */
int cs_b200_session_park_drain(void);

/* ---- search without allocation --------------------------------------
 * No reference counterpart.  cs_gpu_session_run and the enqueue/collect pair
 * may grow the record buffer with cudaMalloc and rerun when more candidates
 * pass the threshold than it holds, and build their result on the host heap.
 * A caller that must not allocate once it is running cannot use them: a
 * real-time pipeline whose latency budget has no room for the device-wide
 * synchronisation a cudaMalloc/cudaFree implies, or a process that reserves
 * all device memory at start-up and hands none out afterwards.
 *
 * This entry point runs the same kernels on a session made earlier by
 * cs_gpu_session_create (whose tables were allocated then) and allocates
 * nothing, on the device or the host: its per-call scratch (spectrum maximum,
 * record counter, error flag, and up to CS_B200_NOALLOC_MAX_RECS records of
 * 16 bytes, about 1 MiB) is a static device array, cleared at the start of
 * each call.  The first call on a device (and the first after a
 * cudaDeviceReset) looks up that array's address and should come before any
 * stream capture.  The scratch is shared by every
 * session on a device, so calls that overlap on the GPU (two streams, two
 * host threads) race and must be serialised by the caller.
 *
 * d_amps: device spectrum (namps float2), or NULL for the session's buffer.
 * out/cap: caller-owned host array for the candidates; also used as staging
 * for the raw records, so cap must be at least the number of records above
 * the threshold.  stream: a cudaStream_t, or NULL for the session stream; the
 * work runs on it after what is already queued on the session stream, and
 * the call waits for it.  The candidates equal those of cs_gpu_session_run in
 * content and order.  Returns 0 and *nout, -1 on a CUDA or kernel error, -2
 * when more than CS_B200_NOALLOC_MAX_RECS records pass the threshold (nothing
 * is returned; raise the threshold or use cs_gpu_session_run), -3 when cap is
 * too small. */
#define CS_B200_NOALLOC_MAX_RECS 65536
int cs_b200_session_search_noalloc(GpuSession *s, const float *d_amps, double threshold,
                                   Candidate *out, long long cap, long long *nout,
                                   void *stream);

#ifdef __cplusplus
}
#endif

#endif
