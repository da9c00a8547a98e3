// The Arrow C data interface at the boundary: a host RecordBatch exported by
// any Arrow implementation (as a struct array) is read in place by
// oxb_import_arrow, and a device batch leaves as one through
// oxb_export_arrow.  The reference's operator hands its backend the same
// buffers (crates/oxidelake-device/src/columns.rs:192-289 extracts values
// and validity from each Arrow array); here the exporter's buffers are read
// directly, so an Arrow producer needs no copy into oxb_column descriptors.
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <string>

#include "internal.h"

namespace oxb {

namespace {

// Whether bits [off, off + n) of an LSB-first bitmap are all set.
bool all_set(const uint8_t* bits, int64_t off, int64_t n) {
    for (int64_t i = 0; i < n; i++)
        if (!((bits[(off + i) >> 3] >> ((off + i) & 7)) & 1)) return false;
    return true;
}

// Bits [off, off + n) of a bitmap, re-based to bit 0.
std::vector<uint8_t> rebase_bits(const uint8_t* bits, int64_t off, int64_t n) {
    std::vector<uint8_t> out((size_t)((n + 7) / 8), 0);
    for (int64_t i = 0; i < n; i++)
        if ((bits[(off + i) >> 3] >> ((off + i) & 7)) & 1) out[(size_t)(i >> 3)] |= (uint8_t)(1u << (i & 7));
    return out;
}

// A primitive Arrow format's column type and value width, or 0.
int primitive_type(const char* fmt, int* width) {
    if (!fmt || fmt[0] == 0 || fmt[1] != 0) return 0;
    switch (fmt[0]) {
        case 'l': *width = 8; return OXB_TYPE_INT64;
        case 'g': *width = 8; return OXB_TYPE_FLOAT64;
        case 'i': *width = 4; return OXB_TYPE_INT32;
        case 'f': *width = 4; return OXB_TYPE_FLOAT32;
        default: return 0;
    }
}

}  // namespace

ArrowImport arrow_import_columns(const ArrowArray* a, const ArrowSchema* sc) {
    if (!a->release || !sc->release) fail(OXB_PLAN, "Arrow array or schema already released");
    if (!sc->format || std::strcmp(sc->format, "+s") != 0)
        fail(OXB_UNSUPPORTED, std::string("Arrow import takes a struct array (a RecordBatch), not format '") +
                                  (sc->format ? sc->format : "") + "'");
    if (a->n_children != sc->n_children) fail(OXB_PLAN, "Arrow array and schema disagree on the column count");
    if (a->length < 0 || a->offset < 0) fail(OXB_PLAN, "negative Arrow length or offset");
    if (a->null_count != 0 && a->n_buffers > 0 && a->buffers && a->buffers[0] &&
        !all_set((const uint8_t*)a->buffers[0], a->offset, a->length))
        fail(OXB_UNSUPPORTED, "null rows in the struct array itself");
    const int64_t rows = a->length;
    ArrowImport imp;
    imp.cols.reserve((size_t)a->n_children);
    imp.rebased.reserve((size_t)a->n_children);
    for (int64_t i = 0; i < a->n_children; i++) {
        const ArrowArray* ca = a->children[i];
        const ArrowSchema* cs = sc->children[i];
        const std::string which = "column " + std::to_string(i);
        if (!ca || !cs) fail(OXB_PLAN, which + " is missing");
        if (ca->dictionary || cs->dictionary) fail(OXB_UNSUPPORTED, which + " is dictionary-encoded");
        const int64_t off = ca->offset + a->offset;  // the parent's offset applies to its children
        if (ca->offset < 0 || ca->length < a->offset + rows) fail(OXB_PLAN, which + " is shorter than the batch");
        oxb_column c{};
        c.length = rows;
        c.dim = 1;
        int width = 0;
        if (const int t = primitive_type(cs->format, &width)) {
            if (ca->n_buffers != 2 || !ca->buffers) fail(OXB_PLAN, which + ": a primitive array has 2 buffers");
            c.type = t;
            c.values = rows > 0 ? (const uint8_t*)ca->buffers[1] + off * width : nullptr;
            if (rows > 0 && !ca->buffers[1]) fail(OXB_PLAN, which + " has no values buffer");
        } else if (cs->format && std::strncmp(cs->format, "+w:", 3) == 0) {
            const long dim = std::strtol(cs->format + 3, nullptr, 10);
            if (dim <= 0 || dim > (1 << 20)) fail(OXB_UNSUPPORTED, which + ": fixed-size list of " + cs->format);
            if (cs->n_children != 1 || ca->n_children != 1 || ca->n_buffers != 1)
                fail(OXB_PLAN, which + ": a fixed-size list has one child and one buffer");
            const ArrowArray* va = ca->children[0];
            const ArrowSchema* vs = cs->children[0];
            int vw = 0;
            if (!va || !vs || primitive_type(vs->format, &vw) != OXB_TYPE_FLOAT32)
                fail(OXB_UNSUPPORTED, which + ": a fixed-size list of other than Float32");
            if (va->n_buffers != 2 || !va->buffers) fail(OXB_PLAN, which + ": list values have 2 buffers");
            const int64_t v0 = va->offset + off * dim;  // the first value of the first row
            if (va->offset < 0 || va->length < (off + rows) * dim)
                fail(OXB_PLAN, which + ": list values shorter than the rows");
            if (va->null_count != 0 && va->buffers[0] && !all_set((const uint8_t*)va->buffers[0], v0, rows * dim))
                fail(OXB_UNSUPPORTED, which + ": null values inside a vector");
            c.type = OXB_TYPE_VECTOR_F32;
            c.dim = (int32_t)dim;
            c.values = rows > 0 ? (const float*)va->buffers[1] + v0 : nullptr;
            if (rows > 0 && !va->buffers[1]) fail(OXB_PLAN, which + " has no values buffer");
        } else {
            fail(OXB_UNSUPPORTED, which + " has Arrow format '" + (cs->format ? cs->format : "") +
                                      "'; Int64, Int32, Float64, Float32 and FixedSizeList<Float32> run on the device");
        }
        const uint8_t* bits = ca->buffers ? (const uint8_t*)ca->buffers[0] : nullptr;
        if (bits && ca->null_count != 0 && rows > 0) {
            if ((off & 7) == 0) {
                c.validity = bits + off / 8;
            } else {
                imp.rebased.push_back(rebase_bits(bits, off, rows));
                c.validity = imp.rebased.back().data();
            }
        }
        imp.cols.push_back(c);
    }
    return imp;
}

namespace {

// Everything an exported array (or schema) tree owns, freed when the last
// struct that refers to it is released: the host copies, the child structs
// and the pointer arrays they point into.
struct ArrayHolder {
    std::atomic<int> refs{0};
    std::vector<std::vector<uint8_t>> data;
    std::vector<ArrowArray> nodes;               // children and list values
    std::vector<ArrowArray*> child_ptrs;         // per node: its children
    std::vector<std::vector<const void*>> bufs;  // per node: its buffers
};

struct SchemaHolder {
    std::atomic<int> refs{0};
    std::vector<std::string> strings;
    std::vector<ArrowSchema> nodes;
    std::vector<ArrowSchema*> child_ptrs;
};

void release_array(ArrowArray* a) {
    if (!a || !a->release) return;
    for (int64_t i = 0; i < a->n_children; i++)
        if (a->children[i] && a->children[i]->release) a->children[i]->release(a->children[i]);
    auto* h = (ArrayHolder*)a->private_data;
    a->release = nullptr;
    if (h->refs.fetch_sub(1) == 1) delete h;
}

void release_schema(ArrowSchema* s) {
    if (!s || !s->release) return;
    for (int64_t i = 0; i < s->n_children; i++)
        if (s->children[i] && s->children[i]->release) s->children[i]->release(s->children[i]);
    auto* h = (SchemaHolder*)s->private_data;
    s->release = nullptr;
    if (h->refs.fetch_sub(1) == 1) delete h;
}

int64_t count_nulls(const std::vector<uint8_t>& bits, int64_t n) {
    int64_t valid = 0;
    for (int64_t i = 0; i < n; i++) valid += (bits[(size_t)(i >> 3)] >> (i & 7)) & 1;
    return n - valid;
}

const char* format_of(int type) {
    switch (type) {
        case OXB_TYPE_INT64: return "l";
        case OXB_TYPE_FLOAT64: return "g";
        case OXB_TYPE_INT32: return "i";
        default: return "f";
    }
}

}  // namespace

void arrow_export_batch(Backend& b, const StreamRef& s, const oxb_batch& batch, const char* const* names,
                        ArrowArray* out_array, ArrowSchema* out_schema, oxb_call_stats& st) {
    const int ncols = (int)batch.cols.size();
    const int64_t rows = batch.rows;
    int nvec = 0;
    for (const Column& c : batch.cols) nvec += c.type == OXB_TYPE_VECTOR_F32;
    const int nnodes = ncols + nvec;  // a vector column adds its values node

    // Host copies of every column, queued together; one synchronization.
    auto ah = std::make_unique<ArrayHolder>();
    ah->data.reserve((size_t)ncols * 2);
    ah->nodes.resize((size_t)nnodes);
    ah->bufs.resize((size_t)nnodes);
    ah->child_ptrs.resize((size_t)nnodes + 1 + ncols);  // per node, then the top struct's children
    std::vector<int> vbits(ncols, -1), vals(ncols, -1);
    for (int i = 0; i < ncols; i++) {
        const Column& c = batch.cols[i];
        const size_t bytes = (size_t)rows * c.width();
        ah->data.emplace_back(bytes ? bytes : 1);
        vals[i] = (int)ah->data.size() - 1;
        if (bytes) download_bytes(b, s, ah->data[vals[i]].data(), c.values, bytes);
        st.bytes_d2h += bytes;
        if (c.validity && rows > 0) {
            ah->data.emplace_back((size_t)(rows + 7) / 8);
            vbits[i] = (int)ah->data.size() - 1;
            OXB_CUDA(cudaMemcpyAsync(ah->data[vbits[i]].data(), c.validity, (size_t)(rows + 7) / 8,
                                     cudaMemcpyDeviceToHost, s->stream));
            st.bytes_d2h += (uint64_t)(rows + 7) / 8;
        }
    }
    OXB_CUDA(cudaStreamSynchronize(s->stream));

    auto sh = std::make_unique<SchemaHolder>();
    sh->strings.reserve((size_t)ncols * 3 + 1);
    sh->nodes.resize((size_t)nnodes);
    sh->child_ptrs.resize((size_t)nnodes + 1 + ncols);
    int next = ncols;  // the values nodes of vector columns follow the columns
    for (int i = 0; i < ncols; i++) {
        const Column& c = batch.cols[i];
        ArrowArray& a = ah->nodes[i];
        ArrowSchema& sc = sh->nodes[i];
        std::memset(&a, 0, sizeof a);
        std::memset(&sc, 0, sizeof sc);
        const bool has_bits = vbits[i] >= 0;
        a.length = rows;
        a.null_count = has_bits ? count_nulls(ah->data[vbits[i]], rows) : 0;
        a.release = release_array;
        a.private_data = ah.get();
        sh->strings.push_back(names && names[i] ? names[i] : "c" + std::to_string(i));
        sc.name = sh->strings.back().c_str();
        sc.flags = ARROW_FLAG_NULLABLE;
        sc.release = release_schema;
        sc.private_data = sh.get();
        if (c.type == OXB_TYPE_VECTOR_F32) {
            ArrowArray& v = ah->nodes[next];
            ArrowSchema& vs = sh->nodes[next];
            std::memset(&v, 0, sizeof v);
            std::memset(&vs, 0, sizeof vs);
            v.length = rows * c.dim;
            v.n_buffers = 2;
            ah->bufs[next] = {nullptr, ah->data[vals[i]].data()};
            v.buffers = ah->bufs[next].data();
            v.release = release_array;
            v.private_data = ah.get();
            vs.format = "f";
            vs.name = "item";
            vs.flags = ARROW_FLAG_NULLABLE;
            vs.release = release_schema;
            vs.private_data = sh.get();
            a.n_buffers = 1;
            ah->bufs[i] = {has_bits ? ah->data[vbits[i]].data() : nullptr};
            a.buffers = ah->bufs[i].data();
            ah->child_ptrs[i] = &v;
            a.n_children = 1;
            a.children = &ah->child_ptrs[i];
            sh->strings.push_back("+w:" + std::to_string(c.dim));
            sc.format = sh->strings.back().c_str();
            sh->child_ptrs[i] = &vs;
            sc.n_children = 1;
            sc.children = &sh->child_ptrs[i];
            next++;
        } else {
            a.n_buffers = 2;
            ah->bufs[i] = {has_bits ? ah->data[vbits[i]].data() : nullptr, ah->data[vals[i]].data()};
            a.buffers = ah->bufs[i].data();
            sc.format = format_of(c.type);
        }
    }
    // The top-level struct array: its children pointers, no buffers of its own.
    static const void* no_bits[1] = {nullptr};
    for (int i = 0; i < ncols; i++) {
        ah->child_ptrs[(size_t)nnodes + 1 + i] = &ah->nodes[i];
        sh->child_ptrs[(size_t)nnodes + 1 + i] = &sh->nodes[i];
    }
    // Every node plus the top struct holds one reference.
    ah->refs = nnodes + 1;
    sh->refs = nnodes + 1;
    std::memset(out_array, 0, sizeof *out_array);
    out_array->length = rows;
    out_array->n_buffers = 1;
    out_array->buffers = no_bits;
    out_array->n_children = ncols;
    out_array->children = ncols ? &ah->child_ptrs[(size_t)nnodes + 1] : nullptr;
    out_array->release = release_array;
    out_array->private_data = ah.release();
    std::memset(out_schema, 0, sizeof *out_schema);
    out_schema->format = "+s";
    out_schema->name = "";
    out_schema->n_children = ncols;
    out_schema->children = ncols ? &sh->child_ptrs[(size_t)nnodes + 1] : nullptr;
    out_schema->release = release_schema;
    out_schema->private_data = sh.release();
    st.rows_in = st.rows_out = (uint64_t)rows;
}

}  // namespace oxb
