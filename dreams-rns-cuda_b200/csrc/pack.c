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

static PyObject *s_blob, *s_K, *s_depth, *s_checkpoint, *s_a0, *s_pcf_init, *s_shadow, *s_q_row,
    *s_p_row, *s_axis, *s_vec;

/* attribute as int64; msg names the overflow (NULL: the default message) */
static int attr_i64(PyObject* o, PyObject* name, int64_t* out, const char* msg) {
    PyObject* v = PyObject_GetAttr(o, name);
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

static int attr_bool(PyObject* o, PyObject* name, int* out) {
    PyObject* v = PyObject_GetAttr(o, name);
    if (!v) return -1;
    int t = PyObject_IsTrue(v);
    Py_DECREF(v);
    if (t < 0) return -1;
    *out = t;
    return 0;
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
    PyObject* index = PyDict_New();          /* blob -> program index */
    PyObject* blobs = PyList_New(0);         /* unique blobs in first-seen order */
    Row* rows = (Row*)calloc(n ? (size_t)n : 1, sizeof(Row));
    I64Vec axis = {0}, vec = {0};
    PyObject* result = NULL;
    if (!index || !blobs || !rows) {
        if (!rows) PyErr_NoMemory();
        goto done;
    }
    for (Py_ssize_t i = 0; i < n; ++i) {
        PyObject* r = items[i];
        Row* w = &rows[i];
        PyObject* b = PyObject_GetAttr(r, s_blob);
        if (!b) goto done;
        if (!PyBytes_Check(b)) {
            Py_DECREF(b);
            PyErr_SetString(PyExc_TypeError, "program blob must be bytes");
            goto done;
        }
        PyObject* j = PyDict_GetItemWithError(index, b);   /* borrowed */
        if (j) {
            w->prog = PyLong_AsLongLong(j);
        } else if (PyErr_Occurred()) {
            Py_DECREF(b);
            goto done;
        } else {
            w->prog = PyList_GET_SIZE(blobs);
            PyObject* k = PyLong_FromLongLong(w->prog);
            if (!k || PyDict_SetItem(index, b, k) || PyList_Append(blobs, b)) {
                Py_XDECREF(k);
                Py_DECREF(b);
                goto done;
            }
            Py_DECREF(k);
        }
        Py_DECREF(b);
        /* axis: every tuple's entries, 4 per program axis */
        PyObject* ax = PyObject_GetAttr(r, s_axis);
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
        PyObject* v = PyObject_GetAttr(r, s_vec);
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
        if (attr_i64(r, s_depth, &w->depth, NULL)) goto done;
        if (w->depth < 0) {
            PyObject* zero = PyLong_FromLong(0);
            if (!zero || PyObject_SetAttr(r, s_depth, zero)) {
                Py_XDECREF(zero);
                goto done;
            }
            Py_DECREF(zero);
            w->depth = 0;
        }
        int pinit = 0, shadow = 0;
        if (attr_i64(r, s_K, &w->K, NULL) || attr_i64(r, s_checkpoint, &w->checkpoint, NULL) ||
            attr_i64(r, s_a0, &w->a0, "a0 outside int64") || attr_bool(r, s_pcf_init, &pinit) ||
            attr_bool(r, s_shadow, &shadow) || attr_i64(r, s_q_row, &w->q_row, NULL) ||
            attr_i64(r, s_p_row, &w->p_row, NULL))
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
        const Py_ssize_t n_prog = PyList_GET_SIZE(blobs);
        size_t blob_bytes = 0;
        for (Py_ssize_t k = 0; k < n_prog; ++k) blob_bytes += (size_t)PyBytes_GET_SIZE(PyList_GET_ITEM(blobs, k));
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
            PyObject* b = PyList_GET_ITEM(blobs, k);
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
    Py_XDECREF(index);
    Py_XDECREF(blobs);
    Py_DECREF(seq);
    return result;
}

static PyMethodDef methods[] = {
    {"pack", pack, METH_O, "Flat C-ABI arrays for a sequence of WalkRequest objects."},
    {NULL, NULL, 0, NULL},
};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_pack", NULL, -1, methods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__pack(void) {
#define INTERN(v, s) if (!(v = PyUnicode_InternFromString(s))) return NULL
    INTERN(s_blob, "blob");
    INTERN(s_K, "K");
    INTERN(s_depth, "depth");
    INTERN(s_checkpoint, "checkpoint");
    INTERN(s_a0, "a0");
    INTERN(s_pcf_init, "pcf_init");
    INTERN(s_shadow, "shadow");
    INTERN(s_q_row, "q_row");
    INTERN(s_p_row, "p_row");
    INTERN(s_axis, "axis");
    INTERN(s_vec, "vec");
#undef INTERN
    return PyModule_Create(&module);
}
