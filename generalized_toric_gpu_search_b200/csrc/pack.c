/* Host-side packing of batches of exponent sets for the max_zeros path.
 *
 * The reference's oracles take a Python list of index lists
 * (kernel_cuda_bp.py:290-323).  Flattening 10^4-10^5 small lists into the
 * int32 index array and int64 offsets the device path reads is a per-item
 * Python loop; this extension does it in C and hands back the two arrays as
 * bytearrays, which the caller views with numpy without a copy.
 *
 *   pack(batch) -> (flat: bytearray of int32, offsets: bytearray of int64, k_max: int,
 *                   bad: bool)
 *
 * batch is a sequence of sequences of ints.  `bad` is True when an index lies
 * outside 0..48; such values are stored as given when they fit int32 and as -1
 * otherwise, so a range check on the flat array still sees them. */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>
#include <string.h>

static PyObject* pack(PyObject* self, PyObject* args) {
  PyObject* batch;
  (void)self;
  if (!PyArg_ParseTuple(args, "O", &batch)) return NULL;
  PyObject* outer = PySequence_Fast(batch, "batch must be a sequence of index sequences");
  if (!outer) return NULL;
  const Py_ssize_t n = PySequence_Fast_GET_SIZE(outer);
  PyObject** sets = PySequence_Fast_ITEMS(outer);
  /* first pass: total size (keeps the inner fast sequences) */
  PyObject** inner = (PyObject**)PyMem_Calloc((size_t)(n > 0 ? n : 1), sizeof(PyObject*));
  if (!inner) {
    Py_DECREF(outer);
    return PyErr_NoMemory();
  }
  Py_ssize_t total = 0, k_max = 0;
  PyObject* result = NULL;
  for (Py_ssize_t i = 0; i < n; ++i) {
    inner[i] = PySequence_Fast(sets[i], "every set must be a sequence of indices");
    if (!inner[i]) goto done;
    const Py_ssize_t k = PySequence_Fast_GET_SIZE(inner[i]);
    total += k;
    if (k > k_max) k_max = k;
  }
  PyObject* flat = PyByteArray_FromStringAndSize(NULL, (total > 0 ? total : 1) * (Py_ssize_t)sizeof(int32_t));
  PyObject* offs = PyByteArray_FromStringAndSize(NULL, (n + 1) * (Py_ssize_t)sizeof(int64_t));
  if (!flat || !offs) {
    Py_XDECREF(flat);
    Py_XDECREF(offs);
    goto done;
  }
  int32_t* f = (int32_t*)PyByteArray_AS_STRING(flat);
  int64_t* o = (int64_t*)PyByteArray_AS_STRING(offs);
  int bad = 0;
  Py_ssize_t pos = 0;
  o[0] = 0;
  for (Py_ssize_t i = 0; i < n; ++i) {
    const Py_ssize_t k = PySequence_Fast_GET_SIZE(inner[i]);
    PyObject** items = PySequence_Fast_ITEMS(inner[i]);
    for (Py_ssize_t j = 0; j < k; ++j) {
      const long v = PyLong_AsLong(items[j]);
      if (v == -1 && PyErr_Occurred()) {
        Py_DECREF(flat);
        Py_DECREF(offs);
        goto done;
      }
      if (v < 0 || v > 48) bad = 1;
      f[pos++] = (v < INT32_MIN || v > INT32_MAX) ? -1 : (int32_t)v;
    }
    o[i + 1] = (int64_t)pos;
  }
  if (total == 0) f[0] = 0;
  result = Py_BuildValue("(NNnO)", flat, offs, k_max, bad ? Py_True : Py_False);
done:
  for (Py_ssize_t i = 0; i < n; ++i) Py_XDECREF(inner[i]);
  PyMem_Free(inner);
  Py_DECREF(outer);
  return result;
}

static PyMethodDef kMethods[] = {
    {"pack", pack, METH_VARARGS, "Flattens a batch of index sequences (int32 flat, int64 offsets)."},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef kModule = {PyModuleDef_HEAD_INIT, "_pack", NULL, -1, kMethods,
                                     NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__pack(void) { return PyModule_Create(&kModule); }
