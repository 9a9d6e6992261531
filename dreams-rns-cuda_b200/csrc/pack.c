/* Request packing for the batched engine (CPython extension dreams_rns._pack).
 *
 * pack(requests) walks a sequence of dreams_rns.engine.WalkRequest objects
 * once and returns the flat arrays of the C ABI: the de-duplicated program
 * blobs and their offsets, one dr_walk_desc per request (the layout of
 * include/dreams_b200.h), the axis parameters followed by the state-vector
 * entries, and the residue offsets.  It is the same computation as the
 * pure-Python _Packed in engine.py, with the same checks and messages; the
 * Python one stays as the reference and is used when this module is absent.
 *
 * Returns (n_programs, offsets, blobs, desc, res_off, cp_off, axis, n_axis,
 * n_res): offsets is uint64[n_programs + 1], desc dr_walk_desc[n], res_off and
 * cp_off int64[n] (cp_off -1 without a checkpoint), axis int64[max(n_axis, 1)],
 * all as bytearrays (so numpy views of them are writable).
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "dreams_b200.h"

typedef struct {
    int64_t* v;
    size_t n, cap;
} I64Vec;

static int vec_push(I64Vec* a, int64_t x) {
    if (a->n == a->cap) {
        size_t cap = a->cap ? 2 * a->cap : 1024;
        int64_t* p = (int64_t*)realloc(a->v, cap * sizeof(int64_t));
        if (!p) {
            PyErr_NoMemory();
            return -1;
        }
        a->v = p;
        a->cap = cap;
    }
    a->v[a->n++] = x;
    return 0;
}

/* the request attributes read, in this order */
enum { A_BLOB, A_K, A_DEPTH, A_CHECKPOINT, A_A0, A_PCF_INIT, A_SHADOW, A_Q_ROW, A_P_ROW, A_AXIS, A_VEC, A_N };
static const char* const attr_names[A_N] = {"blob", "K", "depth", "checkpoint", "a0", "pcf_init",
                                             "shadow", "q_row", "p_row", "axis", "vec"};
static PyObject* names[A_N];

#ifndef Py_T_OBJECT_EX
#include <structmember.h>
#define Py_T_OBJECT_EX T_OBJECT_EX
#endif

/* Attribute reads.  For objects of exactly one type (the type of the first
 * request) whose attributes are __slots__ members and whose attribute lookup
 * is the generic one, a read is the slot's pointer at its offset: the value
 * the generic lookup returns, since a member descriptor is a data descriptor
 * and takes precedence over anything else.  An empty slot, another type or
 * any other kind of attribute goes through PyObject_GetAttr (which raises
 * the AttributeError of an empty slot). */
typedef struct {
    PyTypeObject* type;
    Py_ssize_t off[A_N]; /* -1: no slot read */
} Slots;

static void slots_init(Slots* s, PyTypeObject* t) {
    s->type = t;
    for (int k = 0; k < A_N; ++k) {
        s->off[k] = -1;
        if (!t || t->tp_getattro != PyObject_GenericGetAttr) continue;
        PyObject* d = _PyType_Lookup(t, names[k]); /* borrowed */
        if (d && Py_IS_TYPE(d, &PyMemberDescr_Type)) {
            const PyMemberDef* m = ((PyMemberDescrObject*)d)->d_member;
            if (m->type == Py_T_OBJECT_EX && m->offset > 0) s->off[k] = m->offset;
        }
    }
}

/* new reference to attribute k of o, NULL with an exception set */
static PyObject* get_attr(const Slots* s, PyObject* o, int k) {
    if (Py_TYPE(o) == s->type && s->off[k] > 0) {
        PyObject* v = *(PyObject**)((char*)o + s->off[k]);
        if (v) {
            Py_INCREF(v);
            return v;
        }
    }
    return PyObject_GetAttr(o, names[k]);
}

/* attribute as int64; msg names the overflow (NULL: the default message) */
static int attr_i64(const Slots* s, PyObject* o, int k, int64_t* out, const char* msg) {
    PyObject* v = get_attr(s, o, k);
    if (!v) return -1;
    int overflow = 0;
    long long x = PyLong_AsLongLongAndOverflow(v, &overflow);
    Py_DECREF(v);
    if (overflow) {
        PyErr_SetString(PyExc_OverflowError, msg ? msg : "integer outside int64");
        return -1;
    }
    if (x == -1 && PyErr_Occurred()) return -1;
    *out = (int64_t)x;
    return 0;
}

static int attr_bool(const Slots* s, PyObject* o, int k, int* out) {
    PyObject* v = get_attr(s, o, k);
    if (!v) return -1;
    int t = PyObject_IsTrue(v);
    Py_DECREF(v);
    if (t < 0) return -1;
    *out = t;
    return 0;
}

/* Distinct program blobs by content, in first-seen order: an open-addressing
 * table of bytes objects keyed by their (cached) hash, holding a reference to
 * each distinct blob. */
typedef struct {
    Py_hash_t h;
    PyObject* b;   /* NULL: empty */
    int64_t idx;
} BlobSlot;

typedef struct {
    BlobSlot* slot;
    size_t mask;
    PyObject** uniq;   /* distinct blobs, owned references */
    Py_ssize_t n;
} BlobSet;

static int blobset_init(BlobSet* s, Py_ssize_t max_items) {
    size_t cap = 16;
    while (cap < 2 * (size_t)max_items) cap *= 2;
    s->slot = (BlobSlot*)calloc(cap, sizeof(BlobSlot));
    s->uniq = (PyObject**)malloc((max_items ? (size_t)max_items : 1) * sizeof(PyObject*));
    s->mask = cap - 1;
    s->n = 0;
    if (!s->slot || !s->uniq) {
        PyErr_NoMemory();
        return -1;
    }
    return 0;
}

static void blobset_free(BlobSet* s) {
    for (Py_ssize_t k = 0; k < s->n; ++k) Py_DECREF(s->uniq[k]);
    free(s->slot);
    free(s->uniq);
}

/* index of blob b (bytes), added when new; -1 with an exception set */
static int64_t blobset_index(BlobSet* s, PyObject* b) {
    const Py_hash_t h = PyObject_Hash(b);
    if (h == -1 && PyErr_Occurred()) return -1;
    const Py_ssize_t len = PyBytes_GET_SIZE(b);
    for (size_t i = (size_t)h & s->mask;; i = (i + 1) & s->mask) {
        BlobSlot* e = &s->slot[i];
        if (!e->b) {
            Py_INCREF(b);
            e->h = h;
            e->b = b;
            e->idx = s->n;
            s->uniq[s->n++] = b;
            return e->idx;
        }
        if (e->h == h && (e->b == b || (PyBytes_GET_SIZE(e->b) == len &&
                                         memcmp(PyBytes_AS_STRING(e->b), PyBytes_AS_STRING(b), (size_t)len) == 0)))
            return e->idx;
    }
}

/* append the ints of a sequence to a (overflow: the axis message) */
static int push_ints(I64Vec* a, PyObject* seq, Py_ssize_t* count) {
    PyObject* f = PySequence_Fast(seq, "axis parameters must be sequences of ints");
    if (!f) return -1;
    const Py_ssize_t n = PySequence_Fast_GET_SIZE(f);
    PyObject** it = PySequence_Fast_ITEMS(f);
    for (Py_ssize_t k = 0; k < n; ++k) {
        int overflow = 0;
        long long v = PyLong_AsLongLongAndOverflow(it[k], &overflow);
        if (overflow) {
            Py_DECREF(f);
            PyErr_SetString(PyExc_OverflowError, "axis parameter outside int64");
            return -1;
        }
        if ((v == -1 && PyErr_Occurred()) || vec_push(a, (int64_t)v)) {
            Py_DECREF(f);
            return -1;
        }
    }
    if (count) *count += n;
    Py_DECREF(f);
    return 0;
}

typedef struct {
    int64_t prog, K, depth, checkpoint, a0, flags, q_row, p_row, alen, vlen;
} Row;

static PyObject* pack(PyObject* self, PyObject* arg) {
    (void)self;
    PyObject* seq = PySequence_Fast(arg, "requests must be a sequence");
    if (!seq) return NULL;
    const Py_ssize_t n = PySequence_Fast_GET_SIZE(seq);
    PyObject** items = PySequence_Fast_ITEMS(seq);
    BlobSet blobs = {0};
    Row* rows = (Row*)calloc(n ? (size_t)n : 1, sizeof(Row));
    I64Vec axis = {0}, vec = {0};
    PyObject* result = NULL;
    Slots sl;
    slots_init(&sl, n ? Py_TYPE(items[0]) : NULL);
    if (!rows) {
        PyErr_NoMemory();
        goto done;
    }
    if (blobset_init(&blobs, n)) goto done;
    for (Py_ssize_t i = 0; i < n; ++i) {
        PyObject* r = items[i];
        Row* w = &rows[i];
        PyObject* b = get_attr(&sl, r, A_BLOB);
        if (!b) goto done;
        if (!PyBytes_Check(b)) {
            Py_DECREF(b);
            PyErr_SetString(PyExc_TypeError, "program blob must be bytes");
            goto done;
        }
        w->prog = blobset_index(&blobs, b);
        Py_DECREF(b);
        if (w->prog < 0) goto done;
        /* axis: every tuple's entries, 4 per program axis */
        PyObject* ax = get_attr(&sl, r, A_AXIS);
        if (!ax) goto done;
        PyObject* axf = PySequence_Fast(ax, "axis must be a sequence of tuples");
        Py_DECREF(ax);
        if (!axf) goto done;
        const Py_ssize_t n_ax = PySequence_Fast_GET_SIZE(axf);
        for (Py_ssize_t k = 0; k < n_ax; ++k)
            if (push_ints(&axis, PySequence_Fast_GET_ITEM(axf, k), NULL)) {
                Py_DECREF(axf);
                goto done;
            }
        Py_DECREF(axf);
        w->alen = 4 * (int64_t)n_ax;
        /* state vector */
        PyObject* v = get_attr(&sl, r, A_VEC);
        if (!v) goto done;
        int has_vec = v != Py_None;
        if (has_vec) {
            Py_ssize_t cnt = 0;
            const int rc = push_ints(&vec, v, &cnt);
            Py_DECREF(v);
            if (rc) goto done;
            w->vlen = cnt;
        } else {
            Py_DECREF(v);
        }
        /* scalars; the reference treats a negative depth as no steps */
        if (attr_i64(&sl, r, A_DEPTH, &w->depth, NULL)) goto done;
        if (w->depth < 0) {
            PyObject* zero = PyLong_FromLong(0);
            if (!zero || PyObject_SetAttr(r, names[A_DEPTH], zero)) {
                Py_XDECREF(zero);
                goto done;
            }
            Py_DECREF(zero);
            w->depth = 0;
        }
        int pinit = 0, shadow = 0;
        if (attr_i64(&sl, r, A_K, &w->K, NULL) || attr_i64(&sl, r, A_CHECKPOINT, &w->checkpoint, NULL) ||
            attr_i64(&sl, r, A_A0, &w->a0, "a0 outside int64") || attr_bool(&sl, r, A_PCF_INIT, &pinit) ||
            attr_bool(&sl, r, A_SHADOW, &shadow) || attr_i64(&sl, r, A_Q_ROW, &w->q_row, NULL) ||
            attr_i64(&sl, r, A_P_ROW, &w->p_row, NULL))
            goto done;
        w->flags = (pinit ? DR_WALK_INIT_PCF : 0) | (shadow ? DR_WALK_SHADOW : 0) | (has_vec ? DR_WALK_VEC : 0);
    }
    for (Py_ssize_t i = 0; i < n; ++i)
        if (rows[i].K < 1 || rows[i].K > DR_MAX_K) {
            PyErr_Format(PyExc_ValueError, "K must be in 1..%d", DR_MAX_K);
            goto done;
        }
    for (Py_ssize_t i = 0; i < n; ++i)
        if (rows[i].checkpoint < 0) {
            PyErr_SetString(PyExc_OverflowError, "negative checkpoint");
            goto done;
        }
    {
        const Py_ssize_t n_prog = blobs.n;
        size_t blob_bytes = 0;
        for (Py_ssize_t k = 0; k < n_prog; ++k) blob_bytes += (size_t)PyBytes_GET_SIZE(blobs.uniq[k]);
        const size_t n_axis = axis.n + vec.n;
        PyObject* o_off = PyByteArray_FromStringAndSize(NULL, (Py_ssize_t)(8 * (n_prog + 1)));
        PyObject* o_blob = PyByteArray_FromStringAndSize(NULL, (Py_ssize_t)(blob_bytes ? blob_bytes : 1));
        PyObject* o_desc = PyByteArray_FromStringAndSize(NULL, (Py_ssize_t)(sizeof(dr_walk_desc) * (n ? n : 1)));
        PyObject* o_res = PyByteArray_FromStringAndSize(NULL, (Py_ssize_t)(8 * (n ? n : 1)));
        PyObject* o_cp = PyByteArray_FromStringAndSize(NULL, (Py_ssize_t)(8 * (n ? n : 1)));
        PyObject* o_axis = PyByteArray_FromStringAndSize(NULL, (Py_ssize_t)(8 * (n_axis ? n_axis : 1)));
        if (!o_off || !o_blob || !o_desc || !o_res || !o_cp || !o_axis) {
            Py_XDECREF(o_off); Py_XDECREF(o_blob); Py_XDECREF(o_desc);
            Py_XDECREF(o_res); Py_XDECREF(o_cp); Py_XDECREF(o_axis);
            goto done;
        }
        uint64_t* off = (uint64_t*)PyByteArray_AS_STRING(o_off);
        char* bl = PyByteArray_AS_STRING(o_blob);
        bl[0] = 0;
        off[0] = 0;
        for (Py_ssize_t k = 0; k < n_prog; ++k) {
            PyObject* b = blobs.uniq[k];
            const Py_ssize_t sz = PyBytes_GET_SIZE(b);
            memcpy(bl + off[k], PyBytes_AS_STRING(b), (size_t)sz);
            off[k + 1] = off[k] + (uint64_t)sz;
        }
        dr_walk_desc* desc = (dr_walk_desc*)PyByteArray_AS_STRING(o_desc);
        int64_t* res = (int64_t*)PyByteArray_AS_STRING(o_res);
        int64_t* cp = (int64_t*)PyByteArray_AS_STRING(o_cp);
        memset(desc, 0, sizeof(dr_walk_desc) * (size_t)(n ? n : 1));
        res[0] = 0;
        cp[0] = -1;
        int64_t res_pos = 0, ax_pos = 0, vec_pos = (int64_t)axis.n;
        for (Py_ssize_t i = 0; i < n; ++i) {
            const Row* w = &rows[i];
            dr_walk_desc* d = &desc[i];
            d->program = (uint32_t)w->prog;
            d->K = (uint32_t)w->K;
            d->depth = (uint64_t)w->depth;
            d->checkpoint = (uint64_t)w->checkpoint;
            d->a0 = w->a0;
            d->flags = (uint32_t)w->flags;
            d->q_row = (uint32_t)w->q_row;
            d->p_row = (uint32_t)w->p_row;
            d->axis_offset = (uint64_t)ax_pos;
            d->vec_offset = w->vlen > 0 ? (uint64_t)vec_pos : 0;
            d->res_offset = (uint64_t)res_pos;
            res[i] = res_pos;
            if (w->checkpoint > 0) {
                cp[i] = res_pos + w->K;
                d->cp_res_offset = (uint64_t)cp[i];
            } else {
                cp[i] = -1;
                d->cp_res_offset = 0;
            }
            res_pos += w->K + (w->checkpoint > 0 ? w->K : 0);
            ax_pos += w->alen;
            vec_pos += w->vlen;
        }
        int64_t* axv = (int64_t*)PyByteArray_AS_STRING(o_axis);
        axv[0] = 0;
        if (axis.n) memcpy(axv, axis.v, 8 * axis.n);
        if (vec.n) memcpy(axv + axis.n, vec.v, 8 * vec.n);
        result = Py_BuildValue("(nNNNNNNnL)", n_prog, o_off, o_blob, o_desc, o_res, o_cp, o_axis,
                               (Py_ssize_t)n_axis, (long long)(res_pos > 0 ? res_pos : 1));
    }
done:
    free(rows);
    free(axis.v);
    free(vec.v);
    blobset_free(&blobs);
    Py_DECREF(seq);
    return result;
}

static PyMethodDef methods[] = {
    {"pack", pack, METH_O, "Flat C-ABI arrays for a sequence of WalkRequest objects."},
    {NULL, NULL, 0, NULL},
};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_pack", NULL, -1, methods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__pack(void) {
    for (int k = 0; k < A_N; ++k)
        if (!(names[k] = PyUnicode_InternFromString(attr_names[k]))) return NULL;
    return PyModule_Create(&module);
}
