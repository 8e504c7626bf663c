/*
 * _disptools: NumPy extension with the method table of the reference module
 * (python_c_extension/_disptools.c:532-540 of disptools v0.4.1), backed by
 * the CUDA library libdisptools_b200.so.
 *
 * Same method names, argument order and format strings as the reference
 * built with FLOAT_SIZE=64 (python_c_extension/_disptools.c:42-48).  Changes:
 *  - arrays are checked (dtype, C-contiguity, shape) instead of read through
 *    unchecked PyArray_DATA pointers;
 *  - the GIL is released while the device works;
 *  - None is returned with its reference counted;
 *  - there is no CPU path: gpu_id >= 0 selects that device, gpu_id < 0 the
 *    current one.  `matching` runs volume_matching_3d on the device (the
 *    reference has it on the CPU only, python_c_extension/_disptools.c:368-373);
 *    shape_descriptor is not part of this build and raises
 *    NotImplementedError.
 */
#define PY_SSIZE_T_CLEAN
#define NPY_NO_DEPRECATED_API NPY_1_14_API_VERSION

#include <Python.h>
#include <numpy/arrayobject.h>
#include <string.h>

#include "disptools_b200.h"

static PyObject *raise_library_error(void)
{
    disptools_error_state *err = disptools_get_error();
    PyErr_Format(PyExc_RuntimeError, "%s (%s:%d): %s\n%s", err->function, err->file, err->line,
                 err->message, err->trace);
    return NULL;
}

/* Float triple from a tuple (read_triplet, python_c_extension/_disptools.c:106-123). */
static int read_triplet(PyObject *tuple, double out[3], const char *name)
{
    if (!PyTuple_Check(tuple) || PyTuple_Size(tuple) != 3) {
        PyErr_Format(PyExc_ValueError, "%s must be a tuple of three floats.", name);
        return -1;
    }
    for (int i = 0; i < 3; ++i) {
        out[i] = PyFloat_AsDouble(PyTuple_GetItem(tuple, i));
        if (PyErr_Occurred()) {
            PyErr_Format(PyExc_ValueError, "%s must be a tuple of floats.", name);
            return -1;
        }
    }
    return 0;
}

/* Checks that `obj` is a C-contiguous, aligned, writeable-if-needed ndarray
 * of type `typenum` with `nd` dimensions. */
static PyArrayObject *check_array(PyObject *obj, int typenum, int nd, int writeable, const char *name)
{
    if (!PyArray_Check(obj)) {
        PyErr_Format(PyExc_TypeError, "%s must be a numpy.ndarray", name);
        return NULL;
    }
    PyArrayObject *a = (PyArrayObject *) obj;
    if (PyArray_TYPE(a) != typenum) {
        PyErr_Format(PyExc_TypeError, "%s must have dtype %s", name,
                     typenum == NPY_DOUBLE ? "float64" : "bool");
        return NULL;
    }
    if (PyArray_NDIM(a) != nd) {
        PyErr_Format(PyExc_ValueError, "%s must have %d dimensions", name, nd);
        return NULL;
    }
    if (!PyArray_IS_C_CONTIGUOUS(a) || !PyArray_ISALIGNED(a)) {
        PyErr_Format(PyExc_ValueError, "%s must be C-contiguous and aligned", name);
        return NULL;
    }
    if (writeable && !PyArray_ISWRITEABLE(a)) {
        PyErr_Format(PyExc_ValueError, "%s must be writeable", name);
        return NULL;
    }
    return a;
}

static PyObject *method_get_float_type_size(PyObject *self, PyObject *args)
{
    (void) self;
    (void) args;
    return Py_BuildValue("i", get_float_type_size());
}

/* python_c_extension/_disptools.c:138-167 */
static PyObject *method_regularise(PyObject *self, PyObject *args)
{
    double epsilon;
    PyObject *obj = NULL;
    (void) self;
    if (!PyArg_ParseTuple(args, "Od", &obj, &epsilon)) return NULL;
    PyArrayObject *J = check_array(obj, NPY_DOUBLE, 3, 1, "jacobian");
    if (!J) return NULL;
    const size_t nz = PyArray_DIM(J, 0), ny = PyArray_DIM(J, 1), nx = PyArray_DIM(J, 2);
    double *data = (double *) PyArray_DATA(J);
    Py_BEGIN_ALLOW_THREADS
    regularise(nx, ny, nz, data, epsilon);
    Py_END_ALLOW_THREADS
    if (disptools_has_error()) return raise_library_error();
    Py_RETURN_NONE;
}

static PyObject *method_shape_descriptor(PyObject *self, PyObject *args)
{
    (void) self;
    (void) args;
    PyErr_SetString(PyExc_NotImplementedError,
                    "shape_descriptor is not part of the B200 displacement generator");
    return NULL;
}

/* python_c_extension/_disptools.c:238-274 */
static PyObject *method_jacobian(PyObject *self, PyObject *args)
{
    double spacing[3];
    PyObject *spacing_tuple = NULL, *fobj = NULL, *jobj = NULL;
    (void) self;
    if (!PyArg_ParseTuple(args, "OOO", &spacing_tuple, &fobj, &jobj)) return NULL;
    if (read_triplet(spacing_tuple, spacing, "spacing")) return NULL;
    PyArrayObject *field = check_array(fobj, NPY_DOUBLE, 4, 0, "field");
    if (!field) return NULL;
    PyArrayObject *J = check_array(jobj, NPY_DOUBLE, 3, 1, "jacobian");
    if (!J) return NULL;
    const size_t nz = PyArray_DIM(J, 0), ny = PyArray_DIM(J, 1), nx = PyArray_DIM(J, 2);
    if (PyArray_DIM(field, 0) != 3 || (size_t) PyArray_DIM(field, 1) != nz ||
        (size_t) PyArray_DIM(field, 2) != ny || (size_t) PyArray_DIM(field, 3) != nx) {
        PyErr_SetString(PyExc_ValueError, "field must have shape (3, nz, ny, nx) of the Jacobian");
        return NULL;
    }
    const double *f = (const double *) PyArray_DATA(field);
    double *out = (double *) PyArray_DATA(J);
    Py_BEGIN_ALLOW_THREADS
    jacobian_dynamic(nx, ny, nz, spacing[0], spacing[1], spacing[2], f, out);
    Py_END_ALLOW_THREADS
    if (disptools_has_error()) return raise_library_error();
    Py_RETURN_NONE;
}

/* python_c_extension/_disptools.c:279-422 */
static PyObject *method_displacement(PyObject *self, PyObject *args)
{
    double spacing[3];
    PyObject *spacing_tuple = NULL, *jobj = NULL, *mobj = NULL, *fobj = NULL;
    double epsilon, tolerance, eta, eta_max, alpha, beta, gamma, delta, zeta, theta, iota;
    int strict;
    long it_max;
    const char *algorithm;
    int gpu_id;
    (void) self;
    if (!PyArg_ParseTuple(args, "OOOdddddddddddplOsi", &spacing_tuple, &jobj, &mobj, &epsilon,
                          &tolerance, &eta, &eta_max, &alpha, &beta, &gamma, &delta, &zeta, &theta,
                          &iota, &strict, &it_max, &fobj, &algorithm, &gpu_id))
        return NULL;
    int alg;
    if (!strcmp(algorithm, "gradient")) {
        alg = DTB_ALGORITHM_GRADIENT;
    } else if (!strcmp(algorithm, "greedy")) {
        alg = DTB_ALGORITHM_GREEDY;
    } else if (!strcmp(algorithm, "matching")) {
        alg = DTB_ALGORITHM_MATCHING;
    } else {
        PyErr_Format(PyExc_ValueError, "Invalid algorithm '%s'.", algorithm);
        return NULL;
    }
    if (read_triplet(spacing_tuple, spacing, "spacing")) return NULL;
    PyArrayObject *J = check_array(jobj, NPY_DOUBLE, 3, 0, "jacobian");
    if (!J) return NULL;
    PyArrayObject *mask = check_array(mobj, NPY_BOOL, 3, 0, "mask");
    if (!mask) return NULL;
    PyArrayObject *field = check_array(fobj, NPY_DOUBLE, 4, 1, "field");
    if (!field) return NULL;
    const size_t nz = PyArray_DIM(J, 0), ny = PyArray_DIM(J, 1), nx = PyArray_DIM(J, 2);
    if ((size_t) PyArray_DIM(mask, 0) != nz || (size_t) PyArray_DIM(mask, 1) != ny ||
        (size_t) PyArray_DIM(mask, 2) != nx) {
        PyErr_SetString(PyExc_ValueError, "The shapes of the Jacobian and the mask must agree");
        return NULL;
    }
    if (PyArray_DIM(field, 0) != 3 || (size_t) PyArray_DIM(field, 1) != nz ||
        (size_t) PyArray_DIM(field, 2) != ny || (size_t) PyArray_DIM(field, 3) != nx) {
        PyErr_SetString(PyExc_ValueError, "field must have shape (3, nz, ny, nx) of the Jacobian");
        return NULL;
    }
    if (it_max < 0) {
        PyErr_SetString(PyExc_ValueError, "it_max must be non-negative");
        return NULL;
    }
    if (gpu_id >= 0 && !set_device(gpu_id)) {
        PyErr_Format(PyExc_ValueError, "Cannot set CUDA device %d", gpu_id);
        return NULL;
    }
    const double *Jd = (const double *) PyArray_DATA(J);
    const bool *md = (const bool *) PyArray_DATA(mask);
    double *fd = (double *) PyArray_DATA(field);
    Py_BEGIN_ALLOW_THREADS
    if (alg == DTB_ALGORITHM_GRADIENT)
        generate_displacement_gradient_cuda(nx, ny, nz, spacing[0], spacing[1], spacing[2], Jd, md,
                                            epsilon, tolerance, eta, eta_max, alpha, beta, gamma,
                                            delta, zeta, theta, iota, strict != 0, (size_t) it_max,
                                            fd);
    else if (alg == DTB_ALGORITHM_GREEDY)
        generate_displacement_greedy_cuda(nx, ny, nz, spacing[0], spacing[1], spacing[2], Jd, md,
                                          epsilon, tolerance, eta, eta_max, alpha, beta, gamma,
                                          delta, zeta, theta, iota, strict != 0, (size_t) it_max,
                                          fd);
    else
        volume_matching_3d(nx, ny, nz, spacing[0], spacing[1], spacing[2], Jd, md, epsilon, tolerance,
                           eta, eta_max, alpha, beta, gamma, delta, zeta, theta, iota, strict != 0,
                           (size_t) it_max, fd);
    Py_END_ALLOW_THREADS
    if (disptools_has_error()) return raise_library_error();
    Py_RETURN_NONE;
}

struct module_state {
    PyObject *error;
};
#define GETSTATE(m) ((struct module_state *) PyModule_GetState(m))

static PyObject *error_out(PyObject *self, PyObject *args)
{
    (void) args;
    struct module_state *st = GETSTATE(self);
    PyErr_SetString(st->error, "something bad happened");
    return NULL;
}

static int module_traverse(PyObject *m, visitproc visit, void *arg)
{
    Py_VISIT(GETSTATE(m)->error);
    return 0;
}

static int module_clear(PyObject *m)
{
    Py_CLEAR(GETSTATE(m)->error);
    return 0;
}

static PyMethodDef methods[] = {
    {"error_out", (PyCFunction) error_out, METH_NOARGS, NULL},
    {"get_float_type_size", (PyCFunction) method_get_float_type_size, METH_NOARGS,
     "Get the size of the floating point type.\n\nReturns: int"},
    {"regularise", (PyCFunction) method_regularise, METH_VARARGS,
     "Apply a lower threshold to the Jacobian (in place).\n\n"
     "Parameters\n    Jacobian (numpy.ndarray float64, indices zyx)\n    epsilon (float)\n"},
    {"shape_descriptor", (PyCFunction) method_shape_descriptor, METH_VARARGS,
     "Not available in the B200 build."},
    {"jacobian", (PyCFunction) method_jacobian, METH_VARARGS,
     "Compute the Jacobian of a displacement field.\n\n"
     "Parameters\n    spacing (tuple of three floats)\n"
     "    field (numpy.ndarray float64, indices dzyx)\n"
     "    output Jacobian (numpy.ndarray float64, indices zyx), written in place\n"},
    {"displacement", (PyCFunction) method_displacement, METH_VARARGS,
     "Compute a displacement with given Jacobian (field modified in place).\n\n"
     "Parameters\n    spacing, Jacobian (float64 zyx), mask (bool zyx), epsilon, tolerance, eta,\n"
     "    eta_max, alpha, beta, gamma, delta, zeta, theta, iota, strict, it_max,\n"
     "    field (float64 dzyx, in/out), algorithm ('gradient' or 'greedy'), gpu_id\n"},
    {NULL, NULL, 0, NULL},
};

static struct PyModuleDef moduledef = {
    PyModuleDef_HEAD_INIT, "_disptools",
    "Displacement-field generator (B200 CUDA build) with the interface of disptools' _disptools.",
    sizeof(struct module_state), methods, NULL, module_traverse, module_clear, NULL,
};

PyMODINIT_FUNC PyInit__disptools(void)
{
    PyObject *module = PyModule_Create(&moduledef);
    if (module == NULL) return NULL;
    struct module_state *st = GETSTATE(module);
    st->error = PyErr_NewException("_disptools.Error", NULL, NULL);
    if (st->error == NULL) {
        Py_DECREF(module);
        return NULL;
    }
    import_array();
    return module;
}
