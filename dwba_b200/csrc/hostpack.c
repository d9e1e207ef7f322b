/* Host-side packing of a batch's continuum waves and unpacking of its results (CPython
 * extension, no GPU code).
 *
 * One pass over the (cont_i, cont_f) pairs of a call reads each wave's scalar attributes -- the
 * fields the reference's ContinuumWave carries (k_au, l, idx_match, eta, phase_shift, sigma_l;
 * dwba_matrix_elements.py reads them per pair in radial_ME_all_L) -- and checks and numbers its
 * chi_of_r array, so that the engine's planner gets them as arrays instead of walking thousands of
 * Python objects several times per call:
 *
 *   pack_pairs(pairs, N, ndarray_type) ->
 *       (scalars: bytes of P x 12 doubles (k, l, idx_match, eta, phase_shift, sigma_l of cont_i,
 *                 then of cont_f),
 *        rows_i, rows_f: bytes of P int64 (row of each pair's chi in the batch's function matrix:
 *                 distinct chi objects numbered in order of first appearance, pair by pair, cont_i
 *                 before cont_f -- the order of a matrix whose rows hold the pairs' two waves in
 *                 turn, which then goes to the device as one copy without a gather),
 *        arrays: list of the distinct chi objects in row order,
 *        ptrs: list of the data addresses of the distinct arrays, in row order)
 *   or None when some wave does not qualify (its chi_of_r not exactly an ndarray of N float64
 *   values in C order, or l / k_au missing): the caller then takes its general path.
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>
#include <string.h>

/* attribute names, interned once at import (PyObject_GetAttrString would build each per call) */
enum { A_K, A_L, A_IDX, A_ETA, A_PHASE, A_SIGMA, A_CHI, N_ATTR };
static const char* const attr_names[N_ATTR] = {"k_au", "l", "idx_match", "eta", "phase_shift", "sigma_l", "chi_of_r"};
static PyObject* attr[N_ATTR];

static int get_double(PyObject* o, PyObject* name, double dflt, int required, double* out) {
  PyObject* v = PyObject_GetAttr(o, name);
  if (!v) {
    if (!PyErr_ExceptionMatches(PyExc_AttributeError)) return -1;
    PyErr_Clear();
    if (required) return 1;
    *out = dflt;
    return 0;
  }
  const double d = PyFloat_AsDouble(v);
  Py_DECREF(v);
  if (d == -1.0 && PyErr_Occurred()) return -1;
  *out = d;
  return 0;
}

/* the row of chi (by object identity) in rows_map, numbered on first sight; -1 on error,
 * -2 when chi does not qualify */
static Py_ssize_t chi_row(PyObject* chi, Py_ssize_t N, PyTypeObject* nd, PyObject* rows_map, PyObject* arrays,
                          PyObject* ptrs) {
  if (Py_TYPE(chi) != nd) return -2;
  PyObject* key = PyLong_FromVoidPtr((void*)chi);
  if (!key) return -1;
  PyObject* hit = PyDict_GetItemWithError(rows_map, key);
  if (hit) {
    const Py_ssize_t r = PyLong_AsSsize_t(hit);
    Py_DECREF(key);
    return r;
  }
  if (PyErr_Occurred()) {
    Py_DECREF(key);
    return -1;
  }
  Py_buffer view;
  if (PyObject_GetBuffer(chi, &view, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) != 0) {
    PyErr_Clear();
    Py_DECREF(key);
    return -2;
  }
  const int ok = view.ndim == 1 && view.itemsize == 8 && view.format && strcmp(view.format, "d") == 0 &&
                 view.shape && view.shape[0] == N;
  const int64_t addr = (int64_t)(intptr_t)view.buf;
  PyBuffer_Release(&view);
  if (!ok) {
    Py_DECREF(key);
    return -2;
  }
  const Py_ssize_t r = PyList_GET_SIZE(arrays);
  PyObject* rv = PyLong_FromSsize_t(r);
  PyObject* pv = PyLong_FromLongLong((long long)addr);
  if (!rv || !pv || PyDict_SetItem(rows_map, key, rv) != 0 || PyList_Append(arrays, chi) != 0 ||
      PyList_Append(ptrs, pv) != 0) {
    Py_XDECREF(rv);
    Py_XDECREF(pv);
    Py_DECREF(key);
    return -1;
  }
  Py_DECREF(pv);
  Py_DECREF(rv);
  Py_DECREF(key);
  return r;
}

/* scalars of one wave into s[0..5]; 0 ok, 1 does not qualify, -1 error */
static int wave_scalars(PyObject* w, double* s) {
  int rc;
  if ((rc = get_double(w, attr[A_K], 0.0, 1, &s[0])) != 0) return rc;
  if ((rc = get_double(w, attr[A_L], 0.0, 1, &s[1])) != 0) return rc;
  if ((rc = get_double(w, attr[A_IDX], -1.0, 0, &s[2])) != 0) return rc;
  if ((rc = get_double(w, attr[A_ETA], 0.0, 0, &s[3])) != 0) return rc;
  if ((rc = get_double(w, attr[A_PHASE], 0.0, 0, &s[4])) != 0) return rc;
  if ((rc = get_double(w, attr[A_SIGMA], 0.0, 0, &s[5])) != 0) return rc;
  s[1] = (double)(long long)s[1];
  s[2] = (double)(long long)s[2];
  return 0;
}

static PyObject* pack_pairs(PyObject* self, PyObject* args) {
  (void)self;
  PyObject* pairs;
  Py_ssize_t N;
  PyObject* nd_obj;
  if (!PyArg_ParseTuple(args, "OnO", &pairs, &N, &nd_obj)) return NULL;
  if (!PyType_Check(nd_obj)) {
    PyErr_SetString(PyExc_TypeError, "ndarray_type must be a type");
    return NULL;
  }
  PyTypeObject* nd = (PyTypeObject*)nd_obj;
  PyObject* seq = PySequence_Fast(pairs, "pairs must be a sequence");
  if (!seq) return NULL;
  const Py_ssize_t P = PySequence_Fast_GET_SIZE(seq);
  PyObject* scal = PyBytes_FromStringAndSize(NULL, P * 12 * (Py_ssize_t)sizeof(double));
  PyObject* ri = PyBytes_FromStringAndSize(NULL, P * (Py_ssize_t)sizeof(int64_t));
  PyObject* rf = PyBytes_FromStringAndSize(NULL, P * (Py_ssize_t)sizeof(int64_t));
  PyObject* rows_map = PyDict_New();
  PyObject* arrays = PyList_New(0);
  PyObject* ptrs = PyList_New(0);
  PyObject* result = NULL;
  if (!scal || !ri || !rf || !rows_map || !arrays || !ptrs) goto done;
  {
    double* S = (double*)PyBytes_AS_STRING(scal);
    int64_t* RI = (int64_t*)PyBytes_AS_STRING(ri);
    int64_t* RF = (int64_t*)PyBytes_AS_STRING(rf);
    PyObject** items = PySequence_Fast_ITEMS(seq);
    for (Py_ssize_t p = 0; p < P; ++p) {
      for (int side = 0; side < 2; ++side) {
        PyObject* pr = items[p];
        PyObject* w = NULL;
        if (PyTuple_Check(pr) && PyTuple_GET_SIZE(pr) == 2) {
          w = PyTuple_GET_ITEM(pr, side);
          Py_INCREF(w);
        } else {
          w = PySequence_GetItem(pr, side);
          if (!w) goto done;
        }
        const int rc = wave_scalars(w, S + 12 * p + 6 * side);
        if (rc != 0) {
          Py_DECREF(w);
          if (rc < 0) goto done;
          result = Py_None;
          Py_INCREF(result);
          goto done;
        }
        PyObject* chi = PyObject_GetAttr(w, attr[A_CHI]);
        Py_DECREF(w);
        if (!chi) {
          if (!PyErr_ExceptionMatches(PyExc_AttributeError)) goto done;
          PyErr_Clear();
          result = Py_None;
          Py_INCREF(result);
          goto done;
        }
        const Py_ssize_t r = chi_row(chi, N, nd, rows_map, arrays, ptrs);
        Py_DECREF(chi);
        if (r == -1) goto done;
        if (r == -2) {
          result = Py_None;
          Py_INCREF(result);
          goto done;
        }
        (side == 0 ? RI : RF)[p] = (int64_t)r;
      }
    }
    result = Py_BuildValue("(OOOOO)", scal, ri, rf, arrays, ptrs);
  }
done:
  Py_DECREF(seq);
  Py_XDECREF(scal);
  Py_XDECREF(ri);
  Py_XDECREF(rf);
  Py_XDECREF(rows_map);
  Py_XDECREF(arrays);
  Py_XDECREF(ptrs);
  return result;
}

/* float64 C-contiguous buffer of exactly n values; 0 ok, -1 error (set) */
static int get_values(PyObject* o, Py_ssize_t n, Py_buffer* view) {
  if (PyObject_GetBuffer(o, view, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) != 0) return -1;
  if (view->itemsize != 8 || !view->format || strcmp(view->format, "d") != 0 || view->len != n * 8) {
    PyBuffer_Release(view);
    PyErr_SetString(PyExc_ValueError, "expected a C-contiguous float64 array of T x P x (L_max + 1) values");
    return -1;
  }
  return 0;
}

/* make_results(cls, T, P, nl) -> (results, dicts): results is a list of T lists of P instances of
 * cls, made by object.__new__ with their two fields set by object.__setattr__ (what a frozen
 * dataclass's own __init__ does, without its per-call Python overhead): I_L_direct and
 * I_L_exchange, each a dict with the keys 0..nl-1 and None values; dicts lists those dicts,
 * direct then exchange of each (t, p) in order, for fill_results. The caller makes the skeleton
 * while the device computes and fills in the values when they arrive. */
static PyObject* make_results(PyObject* self, PyObject* args) {
  (void)self;
  PyObject* cls_obj;
  Py_ssize_t T, P, nl;
  if (!PyArg_ParseTuple(args, "Onnn", &cls_obj, &T, &P, &nl)) return NULL;
  if (!PyType_Check(cls_obj) || T < 0 || P < 0 || nl < 1) {
    PyErr_SetString(PyExc_ValueError, "make_results: bad class or sizes");
    return NULL;
  }
  PyTypeObject* cls = (PyTypeObject*)cls_obj;
  PyObject *tmpl = NULL, *empty = NULL, *out = NULL, *dicts = NULL, *n_dir = NULL, *n_exc = NULL, *res = NULL;
  tmpl = PyDict_New();
  empty = PyTuple_New(0);
  n_dir = PyUnicode_InternFromString("I_L_direct");
  n_exc = PyUnicode_InternFromString("I_L_exchange");
  out = PyList_New(T);
  dicts = PyList_New(2 * T * P);
  if (!tmpl || !empty || !n_dir || !n_exc || !out || !dicts) goto done;
  /* keys 0..nl-1 laid out once; each dict is a copy of this template (no resize while filling) */
  for (Py_ssize_t l = 0; l < nl; ++l) {
    PyObject* key = PyLong_FromSsize_t(l);
    const int rc = key ? PyDict_SetItem(tmpl, key, Py_None) : -1;
    Py_XDECREF(key);
    if (rc != 0) goto done;
  }
  for (Py_ssize_t t = 0; t < T; ++t) {
    PyObject* row = PyList_New(P);
    if (!row) goto done;
    PyList_SET_ITEM(out, t, row);
    for (Py_ssize_t p = 0; p < P; ++p) {
      PyObject* obj = PyBaseObject_Type.tp_new(cls, empty, NULL);
      if (!obj) goto done;
      PyList_SET_ITEM(row, p, obj);
      for (int side = 0; side < 2; ++side) {
        PyObject* d = PyDict_Copy(tmpl);
        if (!d) goto done;
        PyList_SET_ITEM(dicts, 2 * (t * P + p) + side, d); /* the list owns the reference */
        if (PyObject_GenericSetAttr(obj, side ? n_exc : n_dir, d) != 0) goto done;
      }
    }
  }
  res = PyTuple_Pack(2, out, dicts);
done:
  Py_XDECREF(tmpl);
  Py_XDECREF(empty);
  Py_XDECREF(n_dir);
  Py_XDECREF(n_exc);
  Py_XDECREF(out);
  Py_XDECREF(dicts);
  return res;
}

/* fill_results(dicts, I_dir, I_exc, nl): the dicts of make_results get their values, {L: I[t, p, L]}
 * as Python floats, from two C-contiguous float64 arrays of T x P x nl values. */
static PyObject* fill_results(PyObject* self, PyObject* args) {
  (void)self;
  PyObject *dicts, *dir_obj, *exc_obj;
  Py_ssize_t nl;
  if (!PyArg_ParseTuple(args, "O!OOn", &PyList_Type, &dicts, &dir_obj, &exc_obj, &nl)) return NULL;
  const Py_ssize_t nd = PyList_GET_SIZE(dicts);
  if (nl < 1 || nd % 2 != 0) {
    PyErr_SetString(PyExc_ValueError, "fill_results: bad sizes");
    return NULL;
  }
  Py_buffer vd, ve;
  if (get_values(dir_obj, (nd / 2) * nl, &vd) != 0) return NULL;
  if (get_values(exc_obj, (nd / 2) * nl, &ve) != 0) {
    PyBuffer_Release(&vd);
    return NULL;
  }
  PyObject* keys[64];
  const Py_ssize_t nk = nl < 64 ? nl : 64; /* keys made once; larger L made per item */
  int ok = 1;
  for (Py_ssize_t l = 0; l < nk; ++l) {
    keys[l] = PyLong_FromSsize_t(l);
    ok &= keys[l] != NULL;
  }
  for (Py_ssize_t i = 0; ok && i < nd; ++i) {
    PyObject* d = PyList_GET_ITEM(dicts, i);
    if (!PyDict_Check(d)) {
      PyErr_SetString(PyExc_TypeError, "fill_results: dicts must hold dicts");
      ok = 0;
      break;
    }
    const double* v = (const double*)((i & 1) ? ve.buf : vd.buf) + (i / 2) * nl;
    for (Py_ssize_t l = 0; l < nl; ++l) {
      PyObject* key = l < nk ? keys[l] : PyLong_FromSsize_t(l);
      PyObject* f = key ? PyFloat_FromDouble(v[l]) : NULL;
      const int rc = f ? PyDict_SetItem(d, key, f) : -1;
      Py_XDECREF(f);
      if (l >= nk) Py_XDECREF(key);
      if (rc != 0) {
        ok = 0;
        break;
      }
    }
  }
  for (Py_ssize_t l = 0; l < nk; ++l) Py_XDECREF(keys[l]);
  PyBuffer_Release(&vd);
  PyBuffer_Release(&ve);
  if (!ok) return NULL;
  Py_RETURN_NONE;
}

/* fill_half(dicts, values, nl, side): dicts[2 i + side] of make_results gets {L: values[i, L]} as
 * Python floats for every i, from a C-contiguous float64 array of (len(dicts) / 2) x nl values (the
 * direct integrals with side 0, the exchange ones with side 1). */
static PyObject* fill_half(PyObject* self, PyObject* args) {
  (void)self;
  PyObject *dicts, *val_obj;
  Py_ssize_t nl;
  int side;
  if (!PyArg_ParseTuple(args, "O!Oni", &PyList_Type, &dicts, &val_obj, &nl, &side)) return NULL;
  const Py_ssize_t nd = PyList_GET_SIZE(dicts);
  if (nl < 1 || nd % 2 != 0 || (side != 0 && side != 1)) {
    PyErr_SetString(PyExc_ValueError, "fill_half: bad sizes or side");
    return NULL;
  }
  Py_buffer vb;
  if (get_values(val_obj, (nd / 2) * nl, &vb) != 0) return NULL;
  PyObject* keys[64];
  const Py_ssize_t nk = nl < 64 ? nl : 64;
  int ok = 1;
  for (Py_ssize_t l = 0; l < nk; ++l) {
    keys[l] = PyLong_FromSsize_t(l);
    ok &= keys[l] != NULL;
  }
  for (Py_ssize_t i = side; ok && i < nd; i += 2) {
    PyObject* d = PyList_GET_ITEM(dicts, i);
    if (!PyDict_Check(d)) {
      PyErr_SetString(PyExc_TypeError, "fill_half: dicts must hold dicts");
      ok = 0;
      break;
    }
    const double* v = (const double*)vb.buf + (i / 2) * nl;
    for (Py_ssize_t l = 0; l < nl; ++l) {
      PyObject* key = l < nk ? keys[l] : PyLong_FromSsize_t(l);
      PyObject* f = key ? PyFloat_FromDouble(v[l]) : NULL;
      const int rc = f ? PyDict_SetItem(d, key, f) : -1;
      Py_XDECREF(f);
      if (l >= nk) Py_XDECREF(key);
      if (rc != 0) {
        ok = 0;
        break;
      }
    }
  }
  for (Py_ssize_t l = 0; l < nk; ++l) Py_XDECREF(keys[l]);
  PyBuffer_Release(&vb);
  if (!ok) return NULL;
  Py_RETURN_NONE;
}

static PyMethodDef methods[] = {
    {"pack_pairs", pack_pairs, METH_VARARGS,
     "pack_pairs(pairs, N, ndarray_type) -> (scalars, rows_i, rows_f, arrays, ptrs) or None"},
    {"make_results", make_results, METH_VARARGS,
     "make_results(cls, T, P, nl) -> (results: T lists of P instances of cls, dicts: their 2 T P field dicts)"},
    {"fill_results", fill_results, METH_VARARGS, "fill_results(dicts, I_dir, I_exc, nl): the values of the dicts"},
    {"fill_half", fill_half, METH_VARARGS,
     "fill_half(dicts, values, nl, side): the direct (side 0) or exchange (side 1) dicts' values"},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_hostpack", NULL, -1, methods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__hostpack(void) {
  for (int i = 0; i < N_ATTR; ++i)
    if (!attr[i] && !(attr[i] = PyUnicode_InternFromString(attr_names[i]))) return NULL;
  return PyModule_Create(&module);
}
