/* cubam_b200: the BAM reader hot path on NVIDIA B200 (sm_100a), as a C ABI.
 *
 * Plain pointers and sizes only.  Every `const uint8_t* / int64_t* ...` data
 * argument is DEVICE memory unless its comment says "host".  `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream).  Every
 * entry point returns CB_OK (0) or a CB_ERR_* code; device-side findings
 * (corrupt data) are written to the summary structs, which live in device
 * memory and are read by the caller after synchronising the stream.
 *
 * Each entry point cites the interface of cubam (LouisFaure/cubam) it
 * replaces, as path:line inside that project.
 */
#ifndef CUBAM_B200_H
#define CUBAM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------- */
enum {
    CB_OK = 0,
    CB_ERR_TRUNCATED = 1,     /* "Truncated BGZF file: the last block is incomplete" (src/cubam/bgzf.py:557,567) */
    CB_ERR_NO_CHAIN = 2,      /* "No valid block or record where one was expected: the data is corrupt" (src/cubam/_kernels.py:688) */
    CB_ERR_CORRUPT_BLOCK = 3, /* "Corrupt BGZF block" (src/cubam/bgzf.py:576,584) */
    CB_ERR_INFLATE = 4,       /* "Corrupt BGZF block: it does not inflate to the size in its trailer" (src/cubam/bgzf.py:611) */
    CB_ERR_CRC = 5,           /* CRC32 of a member differs from its trailer (cubam does not check; docs/reading.md:48-51) */
    CB_ERR_TOO_MANY = 6,      /* "Too many candidates: the data is corrupt" (src/cubam/_kernels.py:671) */
    CB_ERR_CAPACITY = 7,      /* an output or workspace buffer given by the caller is too small */
    CB_ERR_CUDA = 8,          /* a CUDA call failed (cb_last_error() has the text) */
    CB_ERR_ARG = 9,           /* invalid argument */
    CB_ERR_TIMEOUT = 10       /* a serving request's deadline passed before it was served (no kernel of
                                 this library waits on another, so no device wait returns it) */
};

/* One BGZF member to inflate: DEFLATE payload at `in` (in_len bytes), output
 * at out_base + out_off (isize bytes), CRC32 from the member's trailer. */
typedef struct cb_member_job {
    const uint8_t* in;
    int64_t out_off;
    uint32_t in_len;
    uint32_t isize;
    uint32_t crc;
    uint32_t reserved;
} cb_member_job;

/* Result of cb_scan_members (device memory). */
typedef struct cb_scan_summary {
    int64_t n_members;    /* chained members, empty ones included */
    int64_t n_jobs;       /* non-empty members = inflate jobs written */
    int64_t used;         /* compressed bytes used: end of the last chained member */
    int64_t total_out;    /* sum of ISIZE of the jobs */
    int64_t n_candidates; /* header matches before chaining */
    int32_t status;       /* CB_OK or CB_ERR_* */
    int32_t chained;      /* 1 when every candidate was on the chain (no pointer jumping) */
} cb_scan_summary;

/* Result of cb_inflate (device memory). */
typedef struct cb_inflate_summary {
    int32_t status;       /* CB_OK, or the worst CB_ERR_* of the jobs */
    int32_t reserved;
    int64_t n_bad;        /* jobs that failed */
    int64_t first_bad;    /* lowest failing job index, or -1 */
} cb_inflate_summary;

/* Result of cb_record_chain (device memory). */
typedef struct cb_chain_summary {
    int64_t n_records;    /* records on the chain from offset 0 */
    int64_t tail;         /* where the record after the last one starts (0 when there is none) */
    int64_t n_candidates; /* 0 when no offset passes the record predicate, else -1 (not counted) */
    int32_t status;       /* CB_OK, CB_ERR_NO_CHAIN or CB_ERR_CAPACITY */
    int32_t chained;      /* 1 when the parallel tile walks agreed, 0 when the chain was walked serially */
} cb_chain_summary;

/* ---- library ------------------------------------------------------------ */

/* Version string of the library. */
const char* cb_version(void);
/* Text of the last CB_ERR_CUDA / CB_ERR_ARG of the calling thread. */
const char* cb_last_error(void);
/* Number of SMs of the current device (for sizing persistent grids). */
int cb_device_sm_count(void);

/* ---- launch parameters (no counterpart in cubam, whose launch shapes are fixed:
 *      src/cubam/_kernels.py:637-641, and whose chunk size is a fixed policy:
 *      src/cubam/_memory.py:11-23) ---------------------------------------------------------------
 * One value per key for the whole process, read by every later launch; the package's autotuner
 * times candidates on a workload and sets the fastest.  Workspace sizes never depend on them.
 *   CB_PARAM_CHAIN_TILE    bytes per tile of the record chain's walk (a warp walks one, staging it in
 *                          shared memory 8 KiB at a time): a power of two, 2-64 KiB, or 0: 64 KiB,
 *                          less for chunks too small to give 16 tiles per SM (0)
 *   CB_PARAM_INFLATE_FORM  the form cb_inflate runs: 1 member per warp, 2 per lane, 3 split (3)
 *   CB_PARAM_DECODE_ROOT   literal/length root bits of form 3's lane decoder: 6, 7 or 8 (7)
 *   CB_PARAM_COPY_WARPS    warps per CTA of form 3's copy kernel: 2, 3 or 6 with a 16 KiB window per
 *                          warp, 12 with an 8 KiB window, 24 with a 4 KiB window (12)
 *   CB_PARAM_DECODE_STEPS  decode steps of form 3 between lane scheduling rounds: 1-64 (16)
 *   CB_PARAM_DECODE_PREFETCH  lines (128 B) of compressed input form 3's decoder asks L2 for ahead of
 *                          each lane's position: 0-16, 0 = none (4)
 *   CB_PARAM_SPLIT_MIN_JOBS   with CB_PARAM_INFLATE_FORM 3, form 0 runs form 1 for calls of fewer jobs
 *                          (form 3 decodes one member per lane, so it needs many members to fill the GPU):
 *                          0 or more (8192; on 15,456 GEX members form 3 took 16.7 ms, form 1 22.0)
 *   CB_PARAM_COPY_UNITS    DEFLATE units each lane of form 3's copy kernel takes per group: 1 (groups of
 *                          32 units), 2 (64; with 6, 12 or 24 copy warps) or 4 (128; with 6 or 12 copy
 *                          warps, else 2) (2)
 *   CB_PARAM_DECODE_PIPELINE  form 3 in two job ranges, each decoded and then copied on its own stream
 *                          (side streams joined back to the caller's by events), so that one range's
 *                          decode and the other's copy fill the lanes a decode leaves idle at its end:
 *                          0 never, 1 from 65,536 jobs, 2 always; only with the job count given on the
 *                          host (d_n_jobs NULL).  The side streams and events are created by the first
 *                          pipelined call on a device, which should come before any stream capture (1)
 * cb_set_param(key, -1) restores the default; an unknown key or a value out of range is CB_ERR_ARG.
 * cb_get_param returns the current value, -1 for an unknown key. */
enum {
    CB_PARAM_CHAIN_TILE = 1,
    CB_PARAM_INFLATE_FORM = 2,
    CB_PARAM_DECODE_ROOT = 3,
    CB_PARAM_COPY_WARPS = 4,
    CB_PARAM_DECODE_STEPS = 5,
    CB_PARAM_DECODE_PREFETCH = 6,
    CB_PARAM_SPLIT_MIN_JOBS = 7,
    CB_PARAM_COPY_UNITS = 8,
    CB_PARAM_DECODE_PIPELINE = 9
};
int cb_set_param(int key, int64_t value);
int64_t cb_get_param(int key);

/* ---- BGZF member scan: replaces bgzf_candidates + bgzf_sizes + chain + the checks of _inflate_blocks
 *      (src/cubam/_kernels.py:69-89, src/cubam/_kernels.py:662-702, src/cubam/bgzf.py:542-586) ---------- */

/* Workspace bytes cb_scan_members needs for an n-byte buffer. */
size_t cb_scan_workspace_bytes(int64_t n);

/* Scan buf[0:n) (starting at a member) for BGZF members with 128-bit loads and warp
 * ballots, keep the chain from offset 0, check it as the reference does (truncation when
 * `eof`, ISIZE <= 65536, the empty-member rule) and write one job per non-empty member to
 * jobs[0:cap) with out_off = out_base_off + the prefix sum of ISIZE.  The result, including
 * the status, goes to *summary (device). */
int cb_scan_members(const uint8_t* buf, int64_t n, int eof, int64_t out_base_off, cb_member_job* jobs, int64_t cap,
                    cb_scan_summary* summary, void* workspace, size_t workspace_bytes, void* stream);

/* ---- Member scan that allocates nothing (no counterpart in the reference) ----------------------
 * Some callers cannot allocate device memory for a workspace: a serving process whose device memory
 * is owned up front by one pool (RMM, PyTorch's caching allocator) that must not see cudaMalloc
 * behind its back, a caller from another runtime (cgo, JNI) with no device allocator of its own, or
 * a latency-sensitive loop where cudaMalloc/cudaFree would synchronise the device.  This entry point
 * is cb_scan_members with its scratch in a fixed array inside the library instead of a workspace:
 * inputs of at most CB_NOALLOC_SCAN_MAX_BYTES (16 MiB) bytes, about 5.5 MB of scratch that every GPU
 * which loads the library holds until the process exits; larger inputs get CB_ERR_CAPACITY (and
 * cb_last_error() says why) before anything is launched.  The caller still passes the input, the
 * job table and the summary.  The first call on a device looks the array's address up for that
 * device (cudaGetSymbolAddress), so make the first call before any stream capture; that address is
 * kept for the life of the process, so a cudaDeviceReset of a device that has used this entry point
 * is not supported (later calls would use a stale address).  All calls share
 * the one array: calls that overlap on the GPU (other streams, other threads) race on it and must
 * be serialised by the caller; nothing in it needs to start at zero. */
#define CB_NOALLOC_SCAN_MAX_BYTES (16LL << 20)
int cb_scan_members_noalloc(const uint8_t* buf, int64_t n, int eof, int64_t out_base_off, cb_member_job* jobs,
                            int64_t cap, cb_scan_summary* summary, void* stream);

/* ---- Inflate: replaces nvcompBatchedDeflateDecompressAsync and the status/size check
 *      (src/cubam/bgzf.py:587-611); adds the CRC32 check ---------------------------------------- */

/* Workspace bytes of cb_inflate's forms 1 and 2 (form 3 takes cb_inflate_split_workspace_bytes). */
size_t cb_inflate_workspace_bytes(void);

/* Inflate jobs[0:n_jobs) (raw DEFLATE: stored, fixed and dynamic Huffman blocks) into
 * out_base + jobs[i].out_off with persistent grids that take members from a work queue.
 * When d_n_jobs is not NULL the job count is read from device memory (n_jobs is then the
 * capacity).  Each member must give exactly isize bytes; with check_crc its CRC32 must match.
 * job_status (device, may be NULL) gets a code per job.  Runs cb_inflate_form with form 0: the
 * form CB_PARAM_INFLATE_FORM names. */
int cb_inflate(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint8_t* out_base, int check_crc,
               uint32_t* job_status, cb_inflate_summary* summary, void* workspace, size_t workspace_bytes,
               void* stream);

/* cb_inflate with the form given: 1 = one member per warp, 2 = one member per lane (most
 * members in flight), 3 = cb_inflate_split, 0 = CB_PARAM_INFLATE_FORM (form 1 in place of form 3 for
 * fewer than CB_PARAM_SPLIT_MIN_JOBS jobs).  Form 3 runs only with a
 * workspace larger than cb_inflate_workspace_bytes() (sized by cb_inflate_split_workspace_bytes);
 * with the small workspace form 1 runs in its place.  Every form gives the same bytes and the same
 * per-job codes.  No cubam counterpart (cubam has one nvCOMP call, src/cubam/bgzf.py:595). */
int cb_inflate_form(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint8_t* out_base,
                    int check_crc, uint32_t* job_status, cb_inflate_summary* summary, void* workspace,
                    size_t workspace_bytes, int form, void* stream);

/* Members the one-member-per-lane form keeps in flight on the current device (0 on error). */
int64_t cb_inflate_lane_slots(void);

/* ---- Inflate, form 3: the Huffman decode and the copy as two kernels (same contract as cb_inflate,
 *      replacing the same nvCOMP call, src/cubam/bgzf.py:587-611) ---------------------------------
 * k_decode decodes one member per lane (32 members per warp in lock step) into 16-bit units in a
 * token arena inside the workspace (a slot of 2 isize + 8 bytes per job, rounded up to 8); k_copy writes each member
 * with one warp through a shared-memory window (CB_PARAM_COPY_WARPS) and checks its CRC32.
 * out_bytes: the sum of isize over the jobs (or more); a job whose slot does not fit a smaller
 * workspace fails with CB_ERR_CAPACITY. */
size_t cb_inflate_split_workspace_bytes(int64_t n_jobs, int64_t out_bytes);
int cb_inflate_split(const cb_member_job* jobs, int64_t n_jobs, const int64_t* d_n_jobs, uint8_t* out_base,
                     int check_crc, uint32_t* job_status, cb_inflate_summary* summary, void* workspace,
                     size_t workspace_bytes, void* stream);

/* ---- Record chain: replaces record_candidates + record_ends + chain (src/cubam/_kernels.py:250-289,
 *      src/cubam/bam.py:403-418) --------------------------------------------------------------- */

size_t cb_record_chain_workspace_bytes(int64_t n);

/* Offsets of the complete records of data[0:n) on the chain from offset 0, under the reference's
 * record predicate (is_record, src/cubam/_kernels.py:250-278): walked by tiles in parallel and
 * stitched, O(records).  Writes offsets[0:cap) (cap >= n / 37 + 1 always suffices) and *summary.
 * cubam's "Too many candidates" error (more than n/32 + 1024 offsets passing the predicate) is not
 * raised: the walk never tests every offset. */
int cb_record_chain(const uint8_t* data, int64_t n, int32_t n_ref, int64_t* offsets, int64_t cap,
                    cb_chain_summary* summary, void* workspace, size_t workspace_bytes, void* stream);

/* The speculative start of the first record of a shard of a file's records (no counterpart in cubam,
 * which reads a file on one GPU from its start, src/cubam/bam.py:421-446): the first offset o < limit
 * where the record predicate holds and holds for the next `hops` records reached by block_size (or the
 * data ends on the way).  *first (device int64) gets o, or -1 when there is none.  A rank of a
 * sharded decode chains from there while the previous rank is still working, and checks the start
 * once the previous rank's incomplete-record tail arrives. */
int cb_first_record(const uint8_t* data, int64_t n, int32_t n_ref, int64_t limit, int32_t hops, int64_t* first,
                    void* stream);

/* ---- Columns: replaces decode_fixed (src/cubam/_kernels.py:292-319, src/cubam/bam.py:269-288) ---- */

int cb_decode_fixed(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* ref, int32_t* pos,
                    int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos, int32_t* tlen,
                    int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right, void* stream);

/* cb_decode_fixed plus, in the same pass over each record, its aligned length (as
 * cb_aligned_length) and read-name hash (as cb_name_hash), each skipped when its pointer is NULL.
 * Fuses cubam's on-request decoders aligned_length and name_hash (src/cubam/bam.py:325-332,
 * src/cubam/bam.py:341-348) into the record pass, so they do not read the records again. */
int cb_decode_records(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* ref, int32_t* pos,
                      int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos, int32_t* tlen,
                      int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right, int32_t* aligned_length,
                      uint64_t* name_hash, void* stream);

/* The record pass in one launch: the fixed columns (all eleven pointers, or ref == NULL for none),
 * aligned_length, name_hash, n_blocks and n_blocks_split (each skipped when NULL; the last two count
 * the aligned blocks of cb_blocks with split_del 0 and 1, fusing its counting pass,
 * src/cubam/_kernels.py:408-437) and k <= 16 aux tags (k = 0 for none; layout as cb_find_tags), from
 * one read of each record's bytes.  A warp stages the bytes of 32 consecutive
 * records in shared memory with coalesced loads and each lane parses one record; bytes outside the
 * staged window are read from global memory, so any offsets are accepted.  cb_decode_fixed,
 * cb_decode_records and cb_find_tags are this pass with the other outputs left out. */
int cb_decode_columns(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* ref, int32_t* pos,
                      int32_t* end, uint8_t* mapq, uint16_t* flag, int32_t* nref, int32_t* npos, int32_t* tlen,
                      int32_t* l_seq, uint16_t* clip_left, uint16_t* clip_right, int32_t* aligned_length,
                      uint64_t* name_hash, int32_t* n_blocks, int32_t* n_blocks_split, const char* names,
                      int32_t k, uint8_t* type, int64_t* voff, int32_t* vlen, int64_t* value, void* stream);

/* ---- Tags: replaces find_tag, one launch per tag (src/cubam/_kernels.py:334-388, src/cubam/bam.py:184-208).
 * One aux walk per record finds k tags (k <= 16); `names` (host) holds 2k characters.  Output is
 * tag-major: type[t * n + i] etc. --------------------------------------------------------------- */
int cb_find_tags(const uint8_t* data, const int64_t* offsets, int64_t n, const char* names, int32_t k,
                 uint8_t* type, int64_t* voff, int32_t* vlen, int64_t* value, void* stream);

/* ---- On-request decoders (src/cubam/bam.py:221-400, src/cubam/_kernels.py:322-620) -------------- */

/* FNV-1a 64 of read names (name_hash, src/cubam/_kernels.py:322-330). */
int cb_name_hash(const uint8_t* data, const int64_t* offsets, int64_t n, uint64_t* out, void* stream);
/* FNV-1a 64 of spans, 0 where vlen < 0 (hash_spans, src/cubam/_kernels.py:532-540). */
int cb_hash_spans(const uint8_t* data, const int64_t* voff, const int32_t* vlen, int64_t n, uint64_t* out,
                  void* stream);
/* [ACGT]{1,24}(-[0-9]{1,3})? packed in 64 bits (pack_acgt, src/cubam/_kernels.py:544-571). */
int cb_pack_acgt(const uint8_t* data, const int64_t* voff, const int32_t* vlen, int64_t n, uint64_t* out,
                 uint8_t* ok, void* stream);
/* Strings of packed codes at dst_off (unpack_acgt, src/cubam/_kernels.py:607-620). */
int cb_unpack_acgt(const uint64_t* codes, const int64_t* dst_off, int64_t n, uint8_t* chars, void* stream);
/* Aligned bases M/=/X (aligned_len, src/cubam/_kernels.py:391-403). */
int cb_aligned_length(const uint8_t* data, const int64_t* offsets, int64_t n, int32_t* out, void* stream);
/* Aligned blocks, two passes as the reference (blocks, src/cubam/_kernels.py:408-437):
 * fill = 0 counts into cnt; fill = 1 writes rec/start/end from first[i]. */
int cb_blocks(const uint8_t* data, const int64_t* offsets, int64_t n, int split_del, int fill, const int64_t* first,
              int32_t* cnt, int64_t* rec, int32_t* start, int32_t* end, void* stream);
/* Base of read rec[j] at reference position refpos[j] (base_at, src/cubam/_kernels.py:498-529). */
int cb_base_at(const uint8_t* data, const int64_t* offsets, const int64_t* rec, const int32_t* refpos, int64_t m,
               int8_t* out, void* stream);
/* dst[dst_off[i]:+size[i]] = src[src_off[i]:+size[i]] (copy_spans, src/cubam/_kernels.py:34-43). */
int cb_copy_spans(const uint8_t* src, uint8_t* dst, const int64_t* src_off, const int64_t* dst_off,
                  const int64_t* size, int64_t n, void* stream);
/* Record sizes incl. the length field (record_sizes, src/cubam/bam.py:308-315). */
int cb_record_sizes(const uint8_t* data, const int64_t* offsets, int64_t n, int64_t* out, void* stream);

/* ---- BGZF writer: replaces nvcompBatchedDeflateCompressAsync (src/cubam/bgzf.py:292-351, called by
 * _deflate_spans :248 and _bgzf_compress :380), crc32_spans / adler32_spans
 * (src/cubam/_kernels.py:93-158) and bgzf_frame (src/cubam/_kernels.py:161-191) ------------------- */

/* Result of cb_deflate_spans (device memory). */
typedef struct cb_deflate_summary {
    int64_t total;        /* bytes written to out */
    int64_t n_stored;     /* spans written as stored blocks (DEFLATE did not shrink them) */
    int32_t status;       /* CB_OK, CB_ERR_ARG (a span longer than allowed) or CB_ERR_CAPACITY (out too small) */
    int32_t reserved;
} cb_deflate_summary;

/* Workspace bytes of cb_deflate_spans for n spans (no device call). */
size_t cb_deflate_workspace_bytes(int64_t n_spans);

/* Compress the spans data[off[i] : off[i] + size[i]], i < n, each to one raw DEFLATE stream, packed
 * one after another in out: stream i at out_off[i], out_size[i] bytes (both device arrays of n;
 * out_size may be NULL).  With bgzf = 0 a span holds at most 65,536 bytes (the reference's limit,
 * src/cubam/bgzf.py:304); with bgzf = 1 at most 65,280 (BLOCK_DATA) and each stream is framed as a
 * BGZF member (18-byte header with BSIZE, the stream, CRC32, ISIZE; SAMv1 4.1), so out_size[i] =
 * stream + 26.  Each span is written as the smallest of a dynamic-Huffman, a fixed-Huffman and a
 * stored block, so a member always fits BGZF's 64 KiB (the reference's stored fallback,
 * src/cubam/bgzf.py:401).  level: 0 = Huffman coding only, 1 = greedy matching, 2-9 = matching
 * with one position of lazy lookahead.  crc (device, n entries, may be NULL) receives the zlib
 * CRC32 of each span.  out has out_cap bytes; sum(size[i] + 36) always suffices.  Spans must lie
 * inside one device allocation of data.  summary->total is the number of bytes written; when
 * summary->status is not CB_OK nothing is written to out.  The output depends only on the input
 * bytes and the level. */
int cb_deflate_spans(const uint8_t* data, const int64_t* off, const int64_t* size, int64_t n, int level, int bgzf,
                     uint8_t* out, int64_t out_cap, int64_t* out_off, int64_t* out_size, uint32_t* crc,
                     cb_deflate_summary* summary, void* workspace, size_t workspace_bytes, void* stream);

/* zlib CRC32 of each span data[off[i] : off[i] + size[i]] (crc32_spans, src/cubam/_kernels.py:93-141). */
int cb_crc32_spans(const uint8_t* data, const int64_t* off, const int64_t* size, int64_t n, uint32_t* out,
                   void* stream);
/* zlib Adler-32 of each span (adler32_spans, src/cubam/_kernels.py:143-158). */
int cb_adler32_spans(const uint8_t* data, const int64_t* off, const int64_t* size, int64_t n, uint32_t* out,
                     void* stream);

/* ---- Batches: a fixed set of device-resident BAM files decoded by one launch sequence, recordable
 * as one CUDA graph.  cubam decodes a chunk at a time with a host synchronisation per chunk
 * (src/cubam/bgzf.py:625-652, src/cubam/bam.py:421-446); a batch's run issues every file's member
 * scan (jobs into one table), ONE inflate for the members of all files, every file's record chain
 * and every file's record pass (cb_decode_columns), with no host synchronisation. ---------------- */

typedef struct cb_batch cb_batch;  /* opaque */

/* One file's results (device pointers, valid until cb_batch_destroy; rewritten by every run). */
typedef struct cb_batch_file {
    const uint8_t* data;      /* the records: inflated bytes after the BAM header */
    int64_t data_bytes;
    const int64_t* offsets;   /* n_records record offsets into data */
    int64_t n_records;
    int64_t n_members;        /* BGZF members, empty ones included */
    int64_t inflated_bytes;   /* header included */
    int64_t header_bytes;
    int32_t n_ref;
    int32_t k_tags;
    int32_t *ref, *pos, *end;
    uint8_t* mapq;
    uint16_t* flag;
    int32_t *nref, *npos, *tlen, *l_seq;
    uint16_t *clip_left, *clip_right;
    uint8_t* tag_type;        /* k_tags * n_records each, tag-major, as cb_find_tags; NULL for k_tags = 0 */
    int64_t* tag_voff;
    int32_t* tag_vlen;
    int64_t* tag_value;
} cb_batch_file;

/* Plan a batch of n_files BGZF-compressed BAM files, comp[i] (device) of comp_bytes[i] bytes, each a
 * whole file; k <= 16 tags (2k characters in `tags`, host) are decoded with the columns.  Runs the
 * first decode on `stream` to size every buffer (synchronises); the batch owns its device memory.
 * Errors: the reference's status of the failing stage (truncated, corrupt block, inflate, CRC, no
 * chain), CB_ERR_ARG for input that is not BAM. */
int cb_batch_create(const uint8_t* const* comp, const int64_t* comp_bytes, int32_t n_files, const char* tags,
                    int32_t k, int check_crc, void* stream, cb_batch** out);
/* One decode of every file on `stream` (the captured graph when there is one); no synchronisation. */
int cb_batch_run(cb_batch* b, void* stream);
/* Record a run as a CUDA graph on `stream` (not the legacy default stream); later runs replay it. */
int cb_batch_capture(cb_batch* b, void* stream);
/* Synchronise `stream` and check the last run: every device status, and counts equal to the plan. */
int cb_batch_check(cb_batch* b, void* stream);
/* File i's results. */
int cb_batch_file_info(const cb_batch* b, int32_t i, cb_batch_file* out);
/* Inflate jobs of a run (all files), and the inflate form it uses. */
int64_t cb_batch_total_jobs(const cb_batch* b);
int cb_batch_form(const cb_batch* b);
void cb_batch_destroy(cb_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* CUBAM_B200_H */
