// A fixed batch of device-resident BAM files decoded by one launch sequence with no host
// synchronisation, recordable as one CUDA graph: the native form of the batched decoder.
//
// cubam decodes one chunk at a time, one nvCOMP call per chunk with host synchronisations between
// (src/cubam/bgzf.py:625-652, src/cubam/bam.py:421-446).  A batch sizes everything once (create),
// then each run issues, on the caller's stream: every file's member scan writing its inflate jobs
// into its slice of one job table, ONE inflate launch for the members of all files, every file's
// record chain over its records (header skipped), and every file's record pass (columns and tags).
// Nothing in a run waits for the host, so capture records it as a CUDA graph and later runs replay
// it with one launch; check reads every device summary once and compares the counts with the plan.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"

int cb_set_error(cudaError_t e);                       // abi.cu
int cb_set_error_text(int code, const char* text);     // abi.cu

namespace {

struct FileState {
    const uint8_t* comp = nullptr;
    int64_t comp_bytes = 0;
    int64_t n_jobs = 0, job_base = 0, out_base = 0, total_out = 0, n_members = 0;
    int64_t header_bytes = 0, n_records = 0, cap = 0;
    int32_t n_ref = 0;
    int64_t* offsets = nullptr;
    int32_t *ref = nullptr, *pos = nullptr, *end = nullptr, *nref = nullptr, *npos = nullptr, *tlen = nullptr,
            *l_seq = nullptr;
    uint8_t* mapq = nullptr;
    uint16_t *flag = nullptr, *clip_left = nullptr, *clip_right = nullptr;
    uint8_t* tag_type = nullptr;
    int64_t* tag_voff = nullptr;
    int32_t* tag_vlen = nullptr;
    int64_t* tag_value = nullptr;
};

}  // namespace

struct cb_batch {
    std::vector<FileState> files;
    char tags[33] = {0};
    int32_t k = 0;
    int check_crc = 1;
    int64_t total_jobs = 0, total_out = 0;
    int form = 0;
    cb_member_job* jobs = nullptr;
    uint8_t* out = nullptr;
    void* scan_ws = nullptr;
    size_t scan_ws_bytes = 0;
    void* inflate_ws = nullptr;
    size_t inflate_ws_bytes = 0;
    void* chain_ws = nullptr;
    size_t chain_ws_bytes = 0;
    cb_scan_summary* scan_summ = nullptr;     // n_files
    cb_inflate_summary* inflate_summ = nullptr;
    cb_chain_summary* chain_summ = nullptr;   // n_files
    std::vector<void*> allocs;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

template <class T> int dalloc(cb_batch* b, T** p, size_t count) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, count ? count * sizeof(T) : 16);
    if (e != cudaSuccess) return cb_set_error(e);
    b->allocs.push_back(q);
    *p = static_cast<T*>(q);
    return CB_OK;
}

// Little-endian fields of host bytes.
int32_t rd_i32(const uint8_t* p) {
    int32_t v;
    memcpy(&v, p, 4);
    return v;
}

// The size of the BAM header at dev (avail inflated bytes) and its reference count (SAMv1 4.2:
// magic, l_text, text, n_ref, then n_ref of l_name, name, l_ref), read back in growing prefixes.
int header_size(const uint8_t* dev, int64_t avail, cudaStream_t s, int64_t* size, int32_t* n_ref) {
    int64_t want = avail < 65536 ? avail : 65536;
    std::vector<uint8_t> h;
    for (;;) {
        h.resize((size_t)want);
        cudaError_t e = cudaMemcpyAsync(h.data(), dev, (size_t)want, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cb_set_error(e);
        int64_t need = 8;
        bool done = false;
        if (want >= 8) {
            if (memcmp(h.data(), "BAM\1", 4) != 0) return cb_set_error_text(CB_ERR_ARG, "cb_batch_create: not a BAM file");
            const int64_t l_text = rd_i32(h.data() + 4);
            if (l_text < 0) return cb_set_error_text(CB_ERR_ARG, "cb_batch_create: corrupt BAM header");
            need = 8 + l_text + 4;
            if (want >= need) {
                const int32_t nr = rd_i32(h.data() + 8 + l_text);
                if (nr < 0) return cb_set_error_text(CB_ERR_ARG, "cb_batch_create: corrupt BAM header");
                int64_t o = need;
                int32_t r = 0;
                for (; r < nr; r++) {
                    if (o + 4 > want) break;
                    const int64_t l_name = rd_i32(h.data() + o);
                    if (l_name < 1) return cb_set_error_text(CB_ERR_ARG, "cb_batch_create: corrupt BAM header");
                    if (o + 4 + l_name + 4 > want) break;
                    o += 4 + l_name + 4;
                }
                need = o + 8 + 256;
                if (r == nr) {
                    *size = o;
                    *n_ref = nr;
                    done = true;
                }
            }
        }
        if (done) return CB_OK;
        if (want >= avail) return cb_set_error_text(CB_ERR_TRUNCATED, "cb_batch_create: the BAM header is incomplete");
        int64_t nw = want * 2 > need ? want * 2 : need;
        want = nw < avail ? nw : avail;
    }
}

int inflate_ws_for(cb_batch* b) {
    int64_t form = cb_param(CB_PARAM_INFLATE_FORM);
    if (form == 3 && b->total_jobs < cb_param(CB_PARAM_SPLIT_MIN_JOBS)) form = 1;
    b->form = (int)form;
    b->inflate_ws_bytes = form == 3 ? cb_inflate_split_workspace_bytes(b->total_jobs, b->total_out)
                                    : cb_inflate_workspace_bytes();
    if (b->inflate_ws_bytes < 512) b->inflate_ws_bytes = 512;
    uint8_t* p = nullptr;
    const int rc = dalloc(b, &p, b->inflate_ws_bytes);
    b->inflate_ws = p;
    return rc;
}

// Scans (writing jobs) and the inflate: the first half of a run.
int launch_inflate_half(cb_batch* b, cudaStream_t s) {
    for (size_t i = 0; i < b->files.size(); i++) {
        FileState& f = b->files[i];
        const int rc = cb_scan_members(f.comp_bytes ? f.comp : nullptr, f.comp_bytes, 1, f.out_base,
                                       b->jobs + f.job_base, f.n_jobs, b->scan_summ + i, b->scan_ws,
                                       b->scan_ws_bytes, s);
        if (rc != CB_OK) return rc;
    }
    return cb_inflate_form(b->jobs, b->total_jobs, nullptr, b->out, b->check_crc, nullptr, b->inflate_summ,
                           b->inflate_ws, b->inflate_ws_bytes, b->form, s);
}

int launch_chains(cb_batch* b, cudaStream_t s) {
    for (size_t i = 0; i < b->files.size(); i++) {
        FileState& f = b->files[i];
        const int64_t n = f.total_out - f.header_bytes;
        const int rc = cb_record_chain(n ? b->out + f.out_base + f.header_bytes : nullptr, n, f.n_ref, f.offsets,
                                       f.cap, b->chain_summ + i, b->chain_ws, b->chain_ws_bytes, s);
        if (rc != CB_OK) return rc;
    }
    return CB_OK;
}

int launch_records(cb_batch* b, cudaStream_t s) {
    for (size_t i = 0; i < b->files.size(); i++) {
        FileState& f = b->files[i];
        if (!f.n_records) continue;
        const int rc = cb_decode_columns(b->out + f.out_base + f.header_bytes, f.offsets, f.n_records, f.ref, f.pos,
                                         f.end, f.mapq, f.flag, f.nref, f.npos, f.tlen, f.l_seq, f.clip_left,
                                         f.clip_right, nullptr, nullptr, nullptr, nullptr, b->tags, b->k, f.tag_type,
                                         f.tag_voff,
                                         f.tag_vlen, f.tag_value, s);
        if (rc != CB_OK) return rc;
    }
    return CB_OK;
}

int run_eager(cb_batch* b, cudaStream_t s) {
    int rc = launch_inflate_half(b, s);
    if (rc == CB_OK) rc = launch_chains(b, s);
    if (rc == CB_OK) rc = launch_records(b, s);
    return rc;
}

}  // namespace

extern "C" void cb_batch_destroy(cb_batch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (void* p : b->allocs) cudaFree(p);
    delete b;
}

extern "C" int cb_batch_create(const uint8_t* const* comp, const int64_t* comp_bytes, int32_t n_files,
                               const char* tags, int32_t k, int check_crc, void* stream, cb_batch** out) {
    if (!out || n_files < 1 || !comp || !comp_bytes || k < 0 || k > 16 || (k && !tags)) return CB_ERR_ARG;
    *out = nullptr;
    for (int32_t i = 0; i < n_files; i++)
        if (comp_bytes[i] < 0 || (comp_bytes[i] && !comp[i])) return CB_ERR_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cb_batch* b = new (std::nothrow) cb_batch();
    if (!b) return cb_set_error_text(CB_ERR_CAPACITY, "cb_batch_create: out of host memory");
    b->files.resize((size_t)n_files);
    b->k = k;
    b->check_crc = check_crc ? 1 : 0;
    if (k) memcpy(b->tags, tags, (size_t)(2 * k));
    int rc = CB_OK;
    auto fail = [&](int code) {
        cb_batch_destroy(b);
        return code;
    };
    // 1. jobs and inflated bytes of each file: one scan pass with no job capacity
    for (int32_t i = 0; i < n_files; i++) {
        b->files[i].comp = comp[i];
        b->files[i].comp_bytes = comp_bytes[i];
        const size_t w = cb_scan_workspace_bytes(comp_bytes[i]);
        if (w > b->scan_ws_bytes) b->scan_ws_bytes = w;
    }
    uint8_t* sws = nullptr;
    cb_member_job* probe = nullptr;
    if ((rc = dalloc(b, &sws, b->scan_ws_bytes)) || (rc = dalloc(b, &b->scan_summ, (size_t)n_files)) ||
        (rc = dalloc(b, &probe, 1)) || (rc = dalloc(b, &b->inflate_summ, 1)) ||
        (rc = dalloc(b, &b->chain_summ, (size_t)n_files)))
        return fail(rc);
    b->scan_ws = sws;
    std::vector<cb_scan_summary> ss((size_t)n_files);
    for (int32_t i = 0; i < n_files; i++) {
        rc = cb_scan_members(comp_bytes[i] ? comp[i] : nullptr, comp_bytes[i], 1, 0, probe, 0, b->scan_summ + i,
                             b->scan_ws, b->scan_ws_bytes, s);
        if (rc != CB_OK) return fail(rc);
    }
    cudaError_t e = cudaMemcpyAsync(ss.data(), b->scan_summ, sizeof(cb_scan_summary) * n_files, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(cb_set_error(e));
    for (int32_t i = 0; i < n_files; i++) {
        FileState& f = b->files[i];
        if (ss[i].status != CB_OK && ss[i].status != CB_ERR_CAPACITY) return fail(ss[i].status);
        f.n_jobs = ss[i].n_jobs;
        f.n_members = ss[i].n_members;
        f.total_out = ss[i].total_out;
        f.job_base = b->total_jobs;
        f.out_base = b->total_out;
        b->total_jobs += f.n_jobs;
        b->total_out += f.total_out;
    }
    // 2. the job table, the output and the inflate workspace; scans and inflate for real
    if ((rc = dalloc(b, &b->jobs, (size_t)b->total_jobs)) || (rc = dalloc(b, &b->out, (size_t)b->total_out)) ||
        (rc = inflate_ws_for(b)))
        return fail(rc);
    if ((rc = launch_inflate_half(b, s)) != CB_OK) return fail(rc);
    cb_inflate_summary is;
    e = cudaMemcpyAsync(ss.data(), b->scan_summ, sizeof(cb_scan_summary) * n_files, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&is, b->inflate_summ, sizeof(is), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(cb_set_error(e));
    for (int32_t i = 0; i < n_files; i++)
        if (ss[i].status != CB_OK) return fail(ss[i].status);
    if (is.status != CB_OK) return fail(is.status);
    // 3. headers, then the chains with room for every possible record (records are 37 bytes or more)
    for (int32_t i = 0; i < n_files; i++) {
        FileState& f = b->files[i];
        if (!f.total_out) return fail(cb_set_error_text(CB_ERR_TRUNCATED, "cb_batch_create: a file holds no data"));
        if ((rc = header_size(b->out + f.out_base, f.total_out, s, &f.header_bytes, &f.n_ref)) != CB_OK) return fail(rc);
        const int64_t n = f.total_out - f.header_bytes;
        f.cap = n / 37 + 1;
        if ((rc = dalloc(b, &f.offsets, (size_t)f.cap))) return fail(rc);
        const size_t w = cb_record_chain_workspace_bytes(n);
        if (w > b->chain_ws_bytes) b->chain_ws_bytes = w;
    }
    uint8_t* cws = nullptr;
    if ((rc = dalloc(b, &cws, b->chain_ws_bytes))) return fail(rc);
    b->chain_ws = cws;
    if ((rc = launch_chains(b, s)) != CB_OK) return fail(rc);
    std::vector<cb_chain_summary> cs((size_t)n_files);
    e = cudaMemcpyAsync(cs.data(), b->chain_summ, sizeof(cb_chain_summary) * n_files, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(cb_set_error(e));
    // 4. exact columns and tags
    for (int32_t i = 0; i < n_files; i++) {
        FileState& f = b->files[i];
        const int64_t n = f.total_out - f.header_bytes;
        if (n > 0) {
            if (cs[i].status != CB_OK) return fail(cs[i].status);
            if (cs[i].tail != n)
                return fail(cb_set_error_text(CB_ERR_TRUNCATED, "truncated BAM file (incomplete record at the end)"));
        }
        f.n_records = n > 0 ? cs[i].n_records : 0;
        const size_t m = (size_t)f.n_records;
        if ((rc = dalloc(b, &f.ref, m)) || (rc = dalloc(b, &f.pos, m)) || (rc = dalloc(b, &f.end, m)) ||
            (rc = dalloc(b, &f.mapq, m)) || (rc = dalloc(b, &f.flag, m)) || (rc = dalloc(b, &f.nref, m)) ||
            (rc = dalloc(b, &f.npos, m)) || (rc = dalloc(b, &f.tlen, m)) || (rc = dalloc(b, &f.l_seq, m)) ||
            (rc = dalloc(b, &f.clip_left, m)) || (rc = dalloc(b, &f.clip_right, m)))
            return fail(rc);
        if (k && ((rc = dalloc(b, &f.tag_type, m * k)) || (rc = dalloc(b, &f.tag_voff, m * k)) ||
                  (rc = dalloc(b, &f.tag_vlen, m * k)) || (rc = dalloc(b, &f.tag_value, m * k))))
            return fail(rc);
        f.cap = f.n_records > 0 ? f.n_records : 1;
    }
    if ((rc = launch_records(b, s)) != CB_OK) return fail(rc);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(cb_set_error(e));
    *out = b;
    return CB_OK;
}

extern "C" int cb_batch_run(cb_batch* b, void* stream) {
    if (!b) return CB_ERR_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (b->exec) return cb_set_error(cudaGraphLaunch(b->exec, s));
    return run_eager(b, s);
}

extern "C" int cb_batch_capture(cb_batch* b, void* stream) {
    if (!b || !stream) return CB_ERR_ARG;  // the legacy default stream cannot be captured
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cb_set_error(e);
    const int rc = run_eager(b, s);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);
    if (rc != CB_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cb_set_error(e);
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) {
        b->exec = nullptr;
        return cb_set_error(e);
    }
    return CB_OK;
}

extern "C" int cb_batch_check(cb_batch* b, void* stream) {
    if (!b) return CB_ERR_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t nf = b->files.size();
    std::vector<cb_scan_summary> ss(nf);
    std::vector<cb_chain_summary> cs(nf);
    cb_inflate_summary is;
    cudaError_t e = cudaMemcpyAsync(ss.data(), b->scan_summ, sizeof(cb_scan_summary) * nf, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cs.data(), b->chain_summ, sizeof(cb_chain_summary) * nf, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&is, b->inflate_summ, sizeof(is), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cb_set_error(e);
    for (size_t i = 0; i < nf; i++)
        if (ss[i].status != CB_OK) return ss[i].status;
    if (is.status != CB_OK) return is.status;
    for (size_t i = 0; i < nf; i++) {
        const FileState& f = b->files[i];
        if (ss[i].n_jobs != f.n_jobs || ss[i].total_out != f.total_out)
            return cb_set_error_text(CB_ERR_ARG, "cb_batch_check: a file's members differ from the plan");
        if (f.total_out - f.header_bytes > 0) {
            if (cs[i].status != CB_OK) return cs[i].status;
            if (cs[i].n_records != f.n_records || cs[i].tail != f.total_out - f.header_bytes)
                return cb_set_error_text(CB_ERR_ARG, "cb_batch_check: a file's records differ from the plan");
        }
    }
    return CB_OK;
}

extern "C" int cb_batch_file_info(const cb_batch* b, int32_t i, cb_batch_file* v) {
    if (!b || !v || i < 0 || (size_t)i >= b->files.size()) return CB_ERR_ARG;
    const FileState& f = b->files[(size_t)i];
    v->data = b->out + f.out_base + f.header_bytes;
    v->data_bytes = f.total_out - f.header_bytes;
    v->offsets = f.offsets;
    v->n_records = f.n_records;
    v->n_members = f.n_members;
    v->inflated_bytes = f.total_out;
    v->header_bytes = f.header_bytes;
    v->n_ref = f.n_ref;
    v->k_tags = b->k;
    v->ref = f.ref;
    v->pos = f.pos;
    v->end = f.end;
    v->mapq = f.mapq;
    v->flag = f.flag;
    v->nref = f.nref;
    v->npos = f.npos;
    v->tlen = f.tlen;
    v->l_seq = f.l_seq;
    v->clip_left = f.clip_left;
    v->clip_right = f.clip_right;
    v->tag_type = f.tag_type;
    v->tag_voff = f.tag_voff;
    v->tag_vlen = f.tag_vlen;
    v->tag_value = f.tag_value;
    return CB_OK;
}

extern "C" int64_t cb_batch_total_jobs(const cb_batch* b) { return b ? b->total_jobs : -1; }
extern "C" int cb_batch_form(const cb_batch* b) { return b ? b->form : -1; }
