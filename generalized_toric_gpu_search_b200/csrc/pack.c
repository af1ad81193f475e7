/* Host-side packing of batches of exponent sets for the max_zeros path.
 *
 * The reference's oracles take a Python list of index lists
 * (kernel_cuda_bp.py:290-323).  Flattening 10^4-10^5 small lists into the
 * int32 index array and int64 offsets the device path reads is a per-item
 * Python loop; this extension does it in C.
 *
 *   pack(batch) -> (flat: bytearray of int32, offsets: bytearray of int64,
 *                   k_max: int, bad: bool)
 *       hands back the two arrays as bytearrays, which the caller views with
 *       numpy without a copy.
 *   pack_into(batch, flat_addr, flat_cap, off_addr, off_cap)
 *       -> (total: int, k_max: int, bad: bool, done: bool)
 *       writes the same arrays into caller-owned memory (for instance pinned
 *       staging buffers that the host-to-device copy reads directly) at the
 *       given addresses, of flat_cap int32 and off_cap int64 elements.  When
 *       the batch needs more (total > flat_cap or len(batch) + 1 > off_cap) it
 *       returns done = False with the sizes in total and k_max; the arrays'
 *       contents are then unspecified (a first pass may have started them).
 *
 * batch is a sequence of sequences of ints.  `bad` is True when an index lies
 * outside 0..48; such values are stored as given when they fit int32 and as -1
 * otherwise, so a range check on the flat array still sees them. */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>
#include <string.h>

/* The batch as fast sequences: outer, and inner[i] for each set (new
 * references, released by release_batch); total indices and k_max. */
typedef struct {
  PyObject* outer;
  PyObject** inner;
  Py_ssize_t n, total, k_max;
} Batch;

static void release_batch(Batch* b) {
  if (b->inner) {
    for (Py_ssize_t i = 0; i < b->n; ++i) Py_XDECREF(b->inner[i]);
    PyMem_Free(b->inner);
  }
  Py_XDECREF(b->outer);
}

static int collect_batch(PyObject* batch, Batch* b) {
  memset(b, 0, sizeof(*b));
  b->outer = PySequence_Fast(batch, "batch must be a sequence of index sequences");
  if (!b->outer) return -1;
  b->n = PySequence_Fast_GET_SIZE(b->outer);
  PyObject** sets = PySequence_Fast_ITEMS(b->outer);
  b->inner = (PyObject**)PyMem_Calloc((size_t)(b->n > 0 ? b->n : 1), sizeof(PyObject*));
  if (!b->inner) {
    PyErr_NoMemory();
    return -1;
  }
  for (Py_ssize_t i = 0; i < b->n; ++i) {
    if (PyList_CheckExact(sets[i]) || PyTuple_CheckExact(sets[i])) {
      Py_INCREF(sets[i]);  /* already a fast sequence */
      b->inner[i] = sets[i];
    } else {
      b->inner[i] = PySequence_Fast(sets[i], "every set must be a sequence of indices");
      if (!b->inner[i]) return -1;
    }
    const Py_ssize_t k = PySequence_Fast_GET_SIZE(b->inner[i]);
    b->total += k;
    if (k > b->k_max) b->k_max = k;
  }
  return 0;
}

/* Writes the flat indices and offsets; -1 with an exception set when an item
 * is not an int. */
/* One item as a C long: exact ints that fit a machine word (every valid
 * index) are read directly, anything else through PyLong_AsLong (which may
 * call __index__). */
static inline long item_value(PyObject* it) {
#if PY_VERSION_HEX >= 0x030C0000
  if (PyLong_CheckExact(it) && PyUnstable_Long_IsCompact((PyLongObject*)it))
    return (long)PyUnstable_Long_CompactValue((PyLongObject*)it);
#endif
  return PyLong_AsLong(it);
}

static int fill_batch(const Batch* b, int32_t* f, int64_t* o, int* bad) {
  Py_ssize_t pos = 0;
  int any_bad = 0;
  o[0] = 0;
  for (Py_ssize_t i = 0; i < b->n; ++i) {
    const Py_ssize_t k = PySequence_Fast_GET_SIZE(b->inner[i]);
    PyObject** items = PySequence_Fast_ITEMS(b->inner[i]);
    for (Py_ssize_t j = 0; j < k; ++j) {
      const long v = item_value(items[j]);
      if (v == -1 && PyErr_Occurred()) return -1;
      any_bad |= (unsigned long)v > 48ul;
      f[pos++] = (v < INT32_MIN || v > INT32_MAX) ? -1 : (int32_t)v;
    }
    o[i + 1] = (int64_t)pos;
  }
  *bad = any_bad;
  return 0;
}

/* One pass over a list or tuple of lists or tuples of exact ints that fit a
 * machine word (what the drivers pass), straight into the caller's arrays: no
 * size pass, no references taken, and the next sets' objects prefetched (the
 * loop is bound by the latency of reaching each set's items).  No Python code
 * runs inside it, so nothing can change the batch under it.  Returns 1 when
 * the batch is written, 0 when it does not fit the capacities or holds
 * anything else (the caller then takes the general path, which also reports
 * the sizes). */
static int fill_direct(PyObject* batch, int32_t* f, Py_ssize_t fcap, int64_t* o,
                       Py_ssize_t ocap, Py_ssize_t* total, Py_ssize_t* k_max, int* bad) {
#if PY_VERSION_HEX >= 0x030C0000
  PyObject** sets;
  Py_ssize_t n;
  if (PyList_CheckExact(batch)) {
    sets = ((PyListObject*)batch)->ob_item;
    n = PyList_GET_SIZE(batch);
  } else if (PyTuple_CheckExact(batch)) {
    sets = ((PyTupleObject*)batch)->ob_item;
    n = PyTuple_GET_SIZE(batch);
  } else {
    return 0;
  }
  if (n + 1 > ocap) return 0;
  Py_ssize_t pos = 0, km = 0;
  int any_bad = 0;
  o[0] = 0;
  for (Py_ssize_t i = 0; i < n; ++i) {
    if (i + 8 < n) __builtin_prefetch(sets[i + 8]);
    if (i + 4 < n && PyList_CheckExact(sets[i + 4]))
      __builtin_prefetch(((PyListObject*)sets[i + 4])->ob_item);
    PyObject* s = sets[i];
    PyObject** items;
    Py_ssize_t k;
    if (PyList_CheckExact(s)) {
      items = ((PyListObject*)s)->ob_item;
      k = PyList_GET_SIZE(s);
    } else if (PyTuple_CheckExact(s)) {
      items = ((PyTupleObject*)s)->ob_item;
      k = PyTuple_GET_SIZE(s);
    } else {
      return 0;
    }
    if (pos + k > fcap) return 0;
    for (Py_ssize_t j = 0; j < k; ++j) {
      PyObject* it = items[j];
      if (!PyLong_CheckExact(it) || !PyUnstable_Long_IsCompact((PyLongObject*)it)) return 0;
      const long v = (long)PyUnstable_Long_CompactValue((PyLongObject*)it);
      any_bad |= (unsigned long)v > 48ul;
      f[pos + j] = (v < INT32_MIN || v > INT32_MAX) ? -1 : (int32_t)v;
    }
    pos += k;
    if (k > km) km = k;
    o[i + 1] = (int64_t)pos;
  }
  *total = pos;
  *k_max = km;
  *bad = any_bad;
  return 1;
#else
  (void)batch, (void)f, (void)fcap, (void)o, (void)ocap, (void)total, (void)k_max, (void)bad;
  return 0;
#endif
}

static PyObject* pack(PyObject* self, PyObject* args) {
  PyObject* batch;
  (void)self;
  if (!PyArg_ParseTuple(args, "O", &batch)) return NULL;
  Batch b;
  PyObject* result = NULL;
  if (collect_batch(batch, &b) == 0) {
    PyObject* flat =
        PyByteArray_FromStringAndSize(NULL, (b.total > 0 ? b.total : 1) * (Py_ssize_t)sizeof(int32_t));
    PyObject* offs = PyByteArray_FromStringAndSize(NULL, (b.n + 1) * (Py_ssize_t)sizeof(int64_t));
    int bad = 0;
    if (flat && offs) {
      int32_t* f = (int32_t*)PyByteArray_AS_STRING(flat);
      if (b.total == 0) f[0] = 0;
      if (fill_batch(&b, f, (int64_t*)PyByteArray_AS_STRING(offs), &bad) == 0) {
        result = Py_BuildValue("(NNnO)", flat, offs, b.k_max, bad ? Py_True : Py_False);
        flat = offs = NULL;  /* owned by result */
      }
    }
    Py_XDECREF(flat);
    Py_XDECREF(offs);
  }
  release_batch(&b);
  return result;
}

static PyObject* pack_into(PyObject* self, PyObject* args) {
  PyObject* batch;
  unsigned long long flat_addr, off_addr;
  Py_ssize_t flat_cap, off_cap;
  (void)self;
  if (!PyArg_ParseTuple(args, "OKnKn", &batch, &flat_addr, &flat_cap, &off_addr, &off_cap))
    return NULL;
  {
    Py_ssize_t total = 0, k_max = 0;
    int bad = 0;
    if (fill_direct(batch, (int32_t*)(uintptr_t)flat_addr, flat_cap, (int64_t*)(uintptr_t)off_addr,
                    off_cap, &total, &k_max, &bad))
      return Py_BuildValue("(nnOO)", total, k_max, bad ? Py_True : Py_False, Py_True);
  }
  Batch b;
  PyObject* result = NULL;
  if (collect_batch(batch, &b) == 0) {
    if (b.total > flat_cap || b.n + 1 > off_cap) {
      result = Py_BuildValue("(nnOO)", b.total, b.k_max, Py_False, Py_False);
    } else {
      int bad = 0;
      if (fill_batch(&b, (int32_t*)(uintptr_t)flat_addr, (int64_t*)(uintptr_t)off_addr, &bad) == 0)
        result = Py_BuildValue("(nnOO)", b.total, b.k_max, bad ? Py_True : Py_False, Py_True);
    }
  }
  release_batch(&b);
  return result;
}

static PyMethodDef kMethods[] = {
    {"pack", pack, METH_VARARGS, "Flattens a batch of index sequences (int32 flat, int64 offsets)."},
    {"pack_into", pack_into, METH_VARARGS,
     "Flattens a batch of index sequences into caller-owned int32 / int64 arrays."},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef kModule = {PyModuleDef_HEAD_INIT, "_pack", NULL, -1, kMethods,
                                     NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__pack(void) { return PyModule_Create(&kModule); }
