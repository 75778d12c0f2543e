/*
 * Python entry points of the host-buffer Searches (module bm25-npu_b200._hostcall).
 *
 * The Search path through ctypes spends about 5 us per call turning numpy arrays into
 * addresses (ndarray.ctypes) and converting arguments, against a Search of about 100 us.
 * These functions take the arrays through the buffer protocol, check their type and
 * length, release the GIL and call the same C ABI (include/bm25_b200.h): bm25_search
 * and bm25_search_learned.  They return the ABI's status; the caller reads the error
 * message with bm25_last_error as for every other entry point.
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>
#include <string.h>

#include "bm25_b200.h"

/* 'kind' of a buffer's element: 'i' signed integer, 'f' float; with its item size. */
static int TypeIs(const Py_buffer *b, char kind, Py_ssize_t size)
{
    const char *f = b->format ? b->format : "B";
    if (*f == '<' || *f == '=' || *f == '@')
        ++f;
    if (f[0] == '\0' || f[1] != '\0' || b->itemsize != size)
        return 0;
    if (kind == 'f')
        return f[0] == 'f';
    return f[0] == 'i' || f[0] == 'l' || f[0] == 'q';
}

static int Take(PyObject *o, Py_buffer *b, char kind, Py_ssize_t size, Py_ssize_t items, int writable,
                const char *what)
{
    if (PyObject_GetBuffer(o, b, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT | (writable ? PyBUF_WRITABLE : 0)) < 0)
        return -1;
    if (!TypeIs(b, kind, size) || b->len < items * size) {
        PyErr_Format(PyExc_ValueError, "%s must be a C-contiguous %s%zd array of at least %zd items", what,
                     kind == 'f' ? "float" : "int", size * 8, items);
        PyBuffer_Release(b);
        return -1;
    }
    return 0;
}

/* Checks the query batch: offsets int64 [q + 1] whose last entry fits the words (int32). */
static int TakeQueries(PyObject *offsets, PyObject *words, Py_ssize_t q, Py_buffer *ob, Py_buffer *wb)
{
    if (q < 1) {
        PyErr_SetString(PyExc_ValueError, "a Search needs at least one query");
        return -1;
    }
    if (Take(offsets, ob, 'i', 8, q + 1, 0, "offsets") < 0)
        return -1;
    if (Take(words, wb, 'i', 4, 1, 0, "words") < 0) {
        PyBuffer_Release(ob);
        return -1;
    }
    const int64_t last = ((const int64_t *)ob->buf)[q];
    if (last < 0 || last > wb->len / 4) {
        PyErr_SetString(PyExc_ValueError, "offsets[q] exceeds the words given");
        PyBuffer_Release(ob);
        PyBuffer_Release(wb);
        return -1;
    }
    return 0;
}

/* search(handle, offsets, words, q, k, scores, ids) -> status */
static PyObject *Search(PyObject *self, PyObject *args)
{
    unsigned long long handle;
    PyObject *offsets, *words, *scores, *ids;
    Py_ssize_t q, k;
    (void)self;
    if (!PyArg_ParseTuple(args, "KOOnnOO", &handle, &offsets, &words, &q, &k, &scores, &ids))
        return NULL;
    if (k < 1 || k > INT32_MAX || q > INT32_MAX) {
        PyErr_SetString(PyExc_ValueError, "k must be in [1, 2^31) and q below 2^31");
        return NULL;
    }
    Py_buffer ob, wb, sb, ib;
    if (TakeQueries(offsets, words, q, &ob, &wb) < 0)
        return NULL;
    if (Take(scores, &sb, 'f', 4, q * k, 1, "scores") < 0)
        goto fail_q;
    if (Take(ids, &ib, 'i', 4, q * k, 1, "ids") < 0)
        goto fail_s;
    int status;
    Py_BEGIN_ALLOW_THREADS
    status = bm25_search((bm25_handle *)(uintptr_t)handle, (const int64_t *)ob.buf, (const int32_t *)wb.buf,
                         (int64_t)q, (int32_t)k, (float *)sb.buf, (int32_t *)ib.buf);
    Py_END_ALLOW_THREADS
    PyBuffer_Release(&ib);
    PyBuffer_Release(&sb);
    PyBuffer_Release(&wb);
    PyBuffer_Release(&ob);
    return PyLong_FromLong(status);
fail_s:
    PyBuffer_Release(&sb);
fail_q:
    PyBuffer_Release(&wb);
    PyBuffer_Release(&ob);
    return NULL;
}

/* search_learned(handle, offsets, words, q, k, scores, ids, exact) -> status */
static PyObject *SearchLearned(PyObject *self, PyObject *args)
{
    unsigned long long handle;
    PyObject *offsets, *words, *scores, *ids, *exact;
    Py_ssize_t q, k;
    (void)self;
    if (!PyArg_ParseTuple(args, "KOOnnOOO", &handle, &offsets, &words, &q, &k, &scores, &ids, &exact))
        return NULL;
    if (k < 1 || k > INT32_MAX || q > INT32_MAX) {
        PyErr_SetString(PyExc_ValueError, "k must be in [1, 2^31) and q below 2^31");
        return NULL;
    }
    Py_buffer ob, wb, sb, ib, eb;
    if (TakeQueries(offsets, words, q, &ob, &wb) < 0)
        return NULL;
    if (Take(scores, &sb, 'f', 4, q * k, 1, "scores") < 0)
        goto fail_q;
    if (Take(ids, &ib, 'i', 4, q * k, 1, "ids") < 0)
        goto fail_s;
    if (Take(exact, &eb, 'i', 4, q, 1, "exact") < 0)
        goto fail_i;
    int status;
    Py_BEGIN_ALLOW_THREADS
    status = bm25_search_learned((bm25_handle *)(uintptr_t)handle, (const int64_t *)ob.buf,
                                 (const int32_t *)wb.buf, (int64_t)q, (int32_t)k, (float *)sb.buf,
                                 (int32_t *)ib.buf, (int32_t *)eb.buf);
    Py_END_ALLOW_THREADS
    PyBuffer_Release(&eb);
    PyBuffer_Release(&ib);
    PyBuffer_Release(&sb);
    PyBuffer_Release(&wb);
    PyBuffer_Release(&ob);
    return PyLong_FromLong(status);
fail_i:
    PyBuffer_Release(&ib);
fail_s:
    PyBuffer_Release(&sb);
fail_q:
    PyBuffer_Release(&wb);
    PyBuffer_Release(&ob);
    return NULL;
}

static PyMethodDef kMethods[] = {
    {"search", Search, METH_VARARGS, "bm25_search on numpy buffers; returns the status"},
    {"search_learned", SearchLearned, METH_VARARGS, "bm25_search_learned on numpy buffers; returns the status"},
    {NULL, NULL, 0, NULL},
};

static struct PyModuleDef kModule = {PyModuleDef_HEAD_INIT, "_hostcall", NULL, -1, kMethods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__hostcall(void) { return PyModule_Create(&kModule); }
