/*
 * psi_module.c -- the drop-in CPython extension "PSI" over libpsi_b200.
 *
 * Same Python surface as PyPSI's module for its density path:
 *   PSI.Grid(type='cart', n=(32,32,32), bounds=((0,0,0),(1,1,1)), fields=[])
 *   PSI.Mesh(loader, filename=None, pos, vel=None, mass=None, connectivity=None, periodic_box=None)
 *   PSI.voxels(grid, mesh, mode='density', refine_tolerance=1.0, refine_max_lvl=0)
 * with the reference's attributes, defaults, validation order and messages
 * (src/PSI.c:58-279, :367-760, :974-1018).  voxels() forwards to
 * psib_voxels() with the GIL released.  Additions: keyword arguments
 * precision='fp64'|'mixed' and deterministic=False of voxels(), and
 * PSI.last_stats() / PSI.device_count().
 *
 * The 'gadget2' / 'gevolution' loaders read snapshots through
 * psib_load_gadget2 / psib_load_gevolution; mode='annihilation' runs the
 * library's annihilation deposit; PSI.RStarTree(mesh).query(box) and
 * PSI.VDF(mesh, sample_pos, tree, ...) run psib_query_elements and
 * psib_sample_vdf.
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#define NPY_NO_DEPRECATED_API NPY_1_7_API_VERSION
#include <numpy/arrayobject.h>
#include <structmember.h>
#include <string.h>

#include "psi_b200.h"

#define GRID_CART 0
#define GRID_HPRING 1

static psib_stats g_last_stats;

/* ------------------------------------------------------------------ Grid */

typedef struct {
    PyObject_HEAD PyObject *type, *fields, *bounds, *n, *d;
    int ctype;
    int dim;
    int cn[3];
    double window[2][3];
    double cd[3];
    double *cfields[6];
} Grid;

static void pinned_free(PyObject *cap)
{
    psib_host_free(PyCapsule_GetPointer(cap, "psib.pinned"));
}

/* A zeroed float64 array, page-locked when a CUDA device is present so that
 * the host<->device copies of voxels() run at full link speed. */
static PyObject *zeros_f64(int nd, npy_intp *dims)
{
    npy_intp count = 1;
    for (int i = 0; i < nd; ++i) count *= dims[i];
    void *p = (count > 0 && psib_device_count() > 0) ? psib_host_alloc((unsigned long long)count * 8) : NULL;
    if (!p) return PyArray_ZEROS(nd, dims, NPY_FLOAT64, 0);
    memset(p, 0, (size_t)count * 8);
    PyObject *arr = PyArray_SimpleNewFromData(nd, dims, NPY_FLOAT64, p);
    if (!arr) {
        psib_host_free(p);
        return NULL;
    }
    PyObject *cap = PyCapsule_New(p, "psib.pinned", pinned_free);
    if (!cap || PyArray_SetBaseObject((PyArrayObject *)arr, cap) < 0) {
        Py_XDECREF(cap);
        Py_DECREF(arr);
        return NULL;
    }
    return arr;
}

static int set_field(Grid *self, const char *name, int tag, int nd, npy_intp *dims)
{
    PyObject *arr = zeros_f64(nd, dims);
    if (!arr) return -1;
    self->cfields[tag] = (double *)PyArray_DATA((PyArrayObject *)arr);
    int r = PyDict_SetItemString(self->fields, name, arr);
    Py_DECREF(arr);
    return r;
}

/* src/PSI.c:58-246 */
static int Grid_init(Grid *self, PyObject *args, PyObject *kwds)
{
    PyObject *type_in = NULL, *bounds_in = NULL, *n_in = NULL, *fields_in = NULL, *tmp;
    static char *kwlist[] = {"type", "n", "bounds", "fields", NULL};
    if (!PyArg_ParseTupleAndKeywords(args, kwds, "|UOOO", kwlist, &type_in, &n_in, &bounds_in, &fields_in)) return -1;

    if (type_in) {
        const char *t = PyUnicode_AsUTF8(type_in);
        if (strcmp(t, "cart") == 0) self->ctype = GRID_CART;
        else if (strcmp(t, "hpring") == 0) self->ctype = GRID_HPRING;
        else {
            self->ctype = -1;
            PyErr_Format(PyExc_ValueError, "Invalid grid type: %s", t);
            return -1;
        }
        tmp = self->type;
        Py_INCREF(type_in);
        self->type = type_in;
        Py_XDECREF(tmp);
    }
    if (self->ctype == GRID_CART) {
        if (n_in && !PyArg_ParseTuple(n_in, "iii", &self->cn[0], &self->cn[1], &self->cn[2])) {
            PyErr_SetString(PyExc_TypeError, "n must be a tuple containing 3 integers");
            return -1;
        }
        tmp = self->n;
        self->n = Py_BuildValue("(iii)", self->cn[0], self->cn[1], self->cn[2]);
        Py_XDECREF(tmp);
        if (bounds_in && !PyArg_ParseTuple(bounds_in, "(ddd)(ddd)", &self->window[0][0], &self->window[0][1],
                                           &self->window[0][2], &self->window[1][0], &self->window[1][1],
                                           &self->window[1][2])) {
            PyErr_SetString(PyExc_TypeError, "bounds must be a tuple containing two tuples of 3 values each");
            return -1;
        }
        tmp = self->bounds;
        self->bounds = Py_BuildValue("((ddd)(ddd))", self->window[0][0], self->window[0][1], self->window[0][2],
                                     self->window[1][0], self->window[1][1], self->window[1][2]);
        Py_XDECREF(tmp);
        for (int ax = 0; ax < self->dim; ++ax)
            self->cd[ax] = (self->window[1][ax] - self->window[0][ax]) / self->cn[ax];
        tmp = self->d;
        self->d = Py_BuildValue("(ddd)", self->cd[0], self->cd[1], self->cd[2]);
        Py_XDECREF(tmp);
        if (self->cn[0] < 0 || self->cn[1] < 0 || self->cn[2] < 0) {
            PyErr_SetString(PyExc_ValueError, "n must be non-negative");
            return -1;
        }

        npy_intp dims[5] = {self->cn[0], self->cn[1], self->cn[2], 3, 3};
        memset(self->cfields, 0, sizeof(self->cfields));
        if (set_field(self, "m", 0, 3, dims) < 0) return -1;
        if (fields_in && fields_in != Py_None) {
            PyObject *seq = PySequence_Fast(fields_in, "Expected a sequence for fields.");
            if (!seq) return -1;
            Py_ssize_t len = PySequence_Fast_GET_SIZE(seq);
            for (Py_ssize_t i = 0; i < len; ++i) {
                PyObject *it = PySequence_Fast_GET_ITEM(seq, i);
                if (!PyUnicode_Check(it)) {
                    Py_DECREF(seq);
                    PyErr_SetString(PyExc_TypeError, "Field identifiers must be strings");
                    return -1;
                }
                const char *s = PyUnicode_AsUTF8(it);
                int r = 0;
                if (strcmp(s, "m") == 0) r = 0;
                else if (strcmp(s, "x") == 0) r = set_field(self, "x", 1, 4, dims);
                else if (strcmp(s, "v") == 0) r = set_field(self, "v", 2, 4, dims);
                else if (strcmp(s, "xx") == 0) r = set_field(self, "xx", 3, 5, dims);
                else if (strcmp(s, "xv") == 0 || strcmp(s, "vx") == 0) r = set_field(self, "xv", 4, 5, dims);
                else if (strcmp(s, "vv") == 0) r = set_field(self, "vv", 5, 5, dims);
                else {
                    Py_DECREF(seq);
                    PyErr_Format(PyExc_ValueError, "Unrecognized field identifier: %s", s);
                    return -1;
                }
                if (r < 0) {
                    Py_DECREF(seq);
                    return -1;
                }
            }
            Py_DECREF(seq);
            if (self->cfields[3] && !self->cfields[1]) {
                PyErr_SetString(PyExc_ValueError, "Field 'xx' requires you to also provide field 'x'.");
                return -1;
            }
            if (self->cfields[4] && !(self->cfields[2] && self->cfields[1])) {
                PyErr_SetString(PyExc_ValueError, "Field 'xv' requires you to also provide fields 'x' and 'v'.");
                return -1;
            }
            if (self->cfields[5] && !self->cfields[2]) {
                PyErr_SetString(PyExc_ValueError, "Field 'vv' requires you to also provide field 'v'.");
                return -1;
            }
        }
    } else if (self->ctype == GRID_HPRING) {
        PyErr_SetString(PyExc_ValueError, "Grid type hpring is not yet implemented");
        return -1;
    } else {
        PyErr_SetString(PyExc_ValueError, "Invalid grid type");
        return -1;
    }
    return 0;
}

/* src/PSI.c:248-279 */
static PyObject *Grid_new(PyTypeObject *type, PyObject *args, PyObject *kwds)
{
    (void)args;
    (void)kwds;
    Grid *self = (Grid *)type->tp_alloc(type, 0);
    if (!self) return NULL;
    self->ctype = GRID_CART;
    self->dim = 3;
    for (int ax = 0; ax < 3; ++ax) {
        self->cn[ax] = 32;
        self->window[0][ax] = 0.0;
        self->window[1][ax] = 1.0;
        self->cd[ax] = (self->window[1][ax] - self->window[0][ax]) / self->cn[ax];
    }
    self->fields = PyDict_New();
    self->type = PyUnicode_FromString("cart");
    Py_INCREF(Py_None);
    self->bounds = Py_None;
    Py_INCREF(Py_None);
    self->n = Py_None;
    Py_INCREF(Py_None);
    self->d = Py_None;
    return (PyObject *)self;
}

static void Grid_dealloc(Grid *self)
{
    Py_XDECREF(self->type);
    Py_XDECREF(self->fields);
    Py_XDECREF(self->bounds);
    Py_XDECREF(self->n);
    Py_XDECREF(self->d);
    Py_TYPE(self)->tp_free((PyObject *)self);
}

static PyMemberDef Grid_members[] = {
    {"type", T_OBJECT, offsetof(Grid, type), 0, "type"},
    {"fields", T_OBJECT, offsetof(Grid, fields), 0, "fields dict"},
    {"bounds", T_OBJECT, offsetof(Grid, bounds), 0, "lower-left and upper-right corners of the grid"},
    {"n", T_OBJECT, offsetof(Grid, n), 0, "number of gridpoints"},
    {"d", T_OBJECT, offsetof(Grid, d), 0, "grid dx"},
    {NULL, 0, 0, 0, NULL}};

static PyTypeObject GridType = {
    PyVarObject_HEAD_INIT(NULL, 0).tp_name = "PSI.Grid",
    .tp_basicsize = sizeof(Grid),
    .tp_dealloc = (destructor)Grid_dealloc,
    .tp_flags = Py_TPFLAGS_DEFAULT | Py_TPFLAGS_BASETYPE,
    .tp_doc = "Cartesian grid of deposited fields",
    .tp_members = Grid_members,
    .tp_init = (initproc)Grid_init,
    .tp_new = Grid_new,
};

/* ------------------------------------------------------------------ Mesh */

typedef struct {
    PyObject_HEAD PyObject *pos, *vel, *mass, *connectivity, *wrapbox;
    int elemtype, dim, periodic, block;
    long long npart, nelem;
    int nside[3];
    double box[2][3];
} Mesh;

static void swap_ref(PyObject **slot, PyObject *v)
{
    PyObject *t = *slot;
    *slot = v;
    Py_XDECREF(t);
}

/* A C-contiguous view of a float64 / int32 array (copied if not contiguous). */
static PyObject *contig(PyObject *a, int npytype)
{
    return (PyObject *)PyArray_FROM_OTF(a, npytype, NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED);
}

/* src/PSI.c:367-722 */
static int Mesh_init(Mesh *self, PyObject *args, PyObject *kwds)
{
    char *cloader = NULL, *cfile = NULL;
    PyObject *posar = NULL, *velar = NULL, *massar = NULL, *box = NULL, *connar = NULL;
    static char *kwlist[] = {"loader", "filename", "pos", "vel", "mass", "connectivity", "periodic_box", NULL};
    if (!PyArg_ParseTupleAndKeywords(args, kwds, "s|sOOOOO", kwlist, &cloader, &cfile, &posar, &velar, &massar,
                                     &connar, &box))
        return -1;
    if (strcmp(cloader, "array") == 0 || strcmp(cloader, "block") == 0) {
        if (box) {
            if (!PyArg_ParseTuple(box, "(ddd)(ddd)", &self->box[0][0], &self->box[0][1], &self->box[0][2],
                                  &self->box[1][0], &self->box[1][1], &self->box[1][2])) {
                PyErr_SetString(PyExc_TypeError, "periodic_box must be a tuple containing two tuples of 3 values each");
                return -1;
            }
            self->periodic = 1;
        } else {
            self->periodic = 0;
        }
    }
    npy_intp nd[4];
    if (strcmp(cloader, "array") == 0) {
        self->block = 0;
        if (!posar || !PyArray_Check(posar)) {
            PyErr_SetString(PyExc_TypeError, "pos must be a numpy array");
            return -1;
        }
        if (PyArray_TYPE((PyArrayObject *)posar) != NPY_FLOAT64) {
            PyErr_SetString(PyExc_TypeError, "pos must be an array of doubles");
            return -1;
        }
        npy_intp *dt = PyArray_DIMS((PyArrayObject *)posar);
        if (PyArray_NDIM((PyArrayObject *)posar) != 2 || dt[1] != 3) {
            PyErr_SetString(PyExc_TypeError, "pos must be a 2D array with shape (npart, 3)");
            return -1;
        }
        self->dim = 3;
        self->npart = dt[0];
        PyObject *p = contig(posar, NPY_FLOAT64);
        if (!p) return -1;
        swap_ref(&self->pos, p);
        if (!connar || !PyArray_Check(connar)) {
            PyErr_SetString(PyExc_TypeError, "connectivity must be a numpy array");
            return -1;
        }
        if (PyArray_TYPE((PyArrayObject *)connar) != NPY_INT32) {
            PyErr_SetString(PyExc_TypeError, "connectivity must be an array of ints");
            return -1;
        }
        dt = PyArray_DIMS((PyArrayObject *)connar);
        if (PyArray_NDIM((PyArrayObject *)connar) != 2) {
            PyErr_SetString(PyExc_TypeError, "connectivity must be a 2D array with shape (nelem, nverts_per_elem)");
            return -1;
        }
        if (dt[1] != 4 && dt[1] != 8 && dt[1] != 27) {
            PyErr_SetString(PyExc_TypeError, "connectivity must be a 2D array where nverts_per_elem is 4, 8, or 27.");
            return -1;
        }
        self->elemtype = (int)dt[1];
        self->nelem = dt[0];
        PyObject *c = contig(connar, NPY_INT32);
        if (!c) return -1;
        swap_ref(&self->connectivity, c);
        if (velar == NULL) {
            nd[0] = self->npart;
            nd[1] = 3;
            PyObject *v = PyArray_ZEROS(2, nd, NPY_FLOAT64, 0);
            if (!v) return -1;
            swap_ref(&self->vel, v);
        } else if (PyArray_Check(velar)) {
            if (PyArray_TYPE((PyArrayObject *)velar) != NPY_FLOAT64) {
                PyErr_SetString(PyExc_TypeError, "if provided, vel must be an array of doubles");
                return -1;
            }
            dt = PyArray_DIMS((PyArrayObject *)velar);
            if (PyArray_NDIM((PyArrayObject *)velar) != 2 || dt[1] != 3 || dt[0] != self->npart) {
                PyErr_SetString(PyExc_TypeError, "if provided, vel must have the same shape as pos");
                return -1;
            }
            PyObject *v = contig(velar, NPY_FLOAT64);
            if (!v) return -1;
            swap_ref(&self->vel, v);
        } else {
            PyErr_SetString(PyExc_TypeError, "if provided, vel must be a numpy array");
            return -1;
        }
        if (massar == NULL) {
            nd[0] = self->nelem;
            PyObject *m = PyArray_SimpleNew(1, nd, NPY_FLOAT64);
            if (!m) return -1;
            double *mp = (double *)PyArray_DATA((PyArrayObject *)m);
            for (npy_intp i = 0; i < nd[0]; ++i) mp[i] = 1.0;
            swap_ref(&self->mass, m);
        } else if (PyArray_Check(massar)) {
            if (PyArray_TYPE((PyArrayObject *)massar) != NPY_FLOAT64) {
                PyErr_SetString(PyExc_TypeError, "if provided, mass must be an array of doubles");
                return -1;
            }
            dt = PyArray_DIMS((PyArrayObject *)massar);
            if (PyArray_NDIM((PyArrayObject *)massar) != 1 || dt[0] != self->nelem) {
                PyErr_SetString(PyExc_TypeError, "if provided, mass must be a 1D array of length nelem");
                return -1;
            }
            PyObject *m = contig(massar, NPY_FLOAT64);
            if (!m) return -1;
            swap_ref(&self->mass, m);
        } else {
            PyErr_SetString(PyExc_TypeError, "if provided, mass must be a numpy array");
            return -1;
        }
    } else if (strcmp(cloader, "block") == 0) {
        self->block = 1;
        if (!posar || !PyArray_Check(posar)) {
            PyErr_SetString(PyExc_TypeError, "pos must be a numpy array");
            return -1;
        }
        if (PyArray_TYPE((PyArrayObject *)posar) != NPY_FLOAT64) {
            PyErr_SetString(PyExc_TypeError, "pos must be an array of doubles");
            return -1;
        }
        npy_intp *dt = PyArray_DIMS((PyArrayObject *)posar);
        if (PyArray_NDIM((PyArrayObject *)posar) != 4 || dt[3] != 3) {
            PyErr_SetString(PyExc_TypeError, "pos must be a 4D array with shape (nx, ny, nz, 3)");
            return -1;
        }
        self->dim = 3;
        self->npart = dt[0] * dt[1] * dt[2];
        for (int i = 0; i < 3; ++i) self->nside[i] = (int)dt[i];
        PyObject *p = contig(posar, NPY_FLOAT64);
        if (!p) return -1;
        swap_ref(&self->pos, p);
        int ne[3];
        for (int i = 0; i < 3; ++i) ne[i] = self->periodic ? self->nside[i] : self->nside[i] - 1;
        if (ne[0] < 0 || ne[1] < 0 || ne[2] < 0) ne[0] = ne[1] = ne[2] = 0;
        self->nelem = (long long)ne[0] * ne[1] * ne[2];
        self->elemtype = 8;
        if (velar == NULL) {
            nd[0] = self->nside[0];
            nd[1] = self->nside[1];
            nd[2] = self->nside[2];
            nd[3] = 3;
            PyObject *v = PyArray_ZEROS(4, nd, NPY_FLOAT64, 0);
            if (!v) return -1;
            swap_ref(&self->vel, v);
        } else if (PyArray_Check(velar)) {
            if (PyArray_TYPE((PyArrayObject *)velar) != NPY_FLOAT64) {
                PyErr_SetString(PyExc_TypeError, "if provided, vel must be an array of doubles");
                return -1;
            }
            dt = PyArray_DIMS((PyArrayObject *)velar);
            if (PyArray_NDIM((PyArrayObject *)velar) != 4 || dt[3] != 3 || dt[0] != self->nside[0] ||
                dt[1] != self->nside[1] || dt[2] != self->nside[2]) {
                PyErr_SetString(PyExc_TypeError, "if provided, vel must have the same shape as pos");
                return -1;
            }
            PyObject *v = contig(velar, NPY_FLOAT64);
            if (!v) return -1;
            swap_ref(&self->vel, v);
        } else {
            PyErr_SetString(PyExc_TypeError, "if provided, vel must be a numpy array");
            return -1;
        }
        if (massar == NULL) {
            nd[0] = ne[0];
            nd[1] = ne[1];
            nd[2] = ne[2];
            PyObject *m = PyArray_SimpleNew(3, nd, NPY_FLOAT64);
            if (!m) return -1;
            double *mp = (double *)PyArray_DATA((PyArrayObject *)m);
            for (long long i = 0; i < self->nelem; ++i) mp[i] = 1.0;
            swap_ref(&self->mass, m);
        } else if (PyArray_Check(massar)) {
            if (PyArray_TYPE((PyArrayObject *)massar) != NPY_FLOAT64) {
                PyErr_SetString(PyExc_TypeError, "if provided, mass must be an array of doubles");
                return -1;
            }
            dt = PyArray_DIMS((PyArrayObject *)massar);
            if (PyArray_NDIM((PyArrayObject *)massar) != 3 || dt[0] != ne[0] || dt[1] != ne[1] || dt[2] != ne[2]) {
                PyErr_SetString(PyExc_TypeError,
                                "if provided, mass must be a 3D array of shape (nelemx, nelemy, nelemz)");
                return -1;
            }
            PyObject *m = contig(massar, NPY_FLOAT64);
            if (!m) return -1;
            swap_ref(&self->mass, m);
        } else {
            PyErr_SetString(PyExc_TypeError, "if provided, mass must be a numpy array");
            return -1;
        }
        /* connectivity of the block (src/PSI.c:636-656), kept as an attribute;
         * voxels() passes the lattice shape instead of this array */
        nd[0] = (npy_intp)self->nelem;
        nd[1] = 8;
        PyObject *c = PyArray_SimpleNew(2, nd, NPY_INT32);
        if (!c) return -1;
        int *cp = (int *)PyArray_DATA((PyArrayObject *)c);
        const int *ns = self->nside;
        for (int i = 0; i < ne[0]; ++i)
            for (int j = 0; j < ne[1]; ++j)
                for (int k = 0; k < ne[2]; ++k) {
                    long long el = ((long long)ne[1] * i + j) * ne[2] + k;
                    for (int ii = 0; ii < 2; ++ii)
                        for (int jj = 0; jj < 2; ++jj)
                            for (int kk = 0; kk < 2; ++kk)
                                cp[8 * el + 4 * ii + 2 * jj + kk] =
                                    ns[1] * ns[2] * ((i + ii) % ns[0]) + ns[2] * ((j + jj) % ns[1]) + ((k + kk) % ns[2]);
                }
        swap_ref(&self->connectivity, c);
    } else if (strcmp(cloader, "gadget2") == 0 || strcmp(cloader, "gevolution") == 0) {
        /* src/PSI.c:659-709: peek at the header, allocate, then load */
        long long np = 0;
        double boxsize = 0.0;
        if (!cfile || psib_peek_gadget2(cfile, &np, &boxsize) != PSIB_OK || np < 0) {
            PyErr_Format(PyExc_ValueError, "Bad file name: %s", cfile ? cfile : "(none)");
            return -1;
        }
        nd[0] = (npy_intp)np;
        nd[1] = 3;
        PyObject *p = PyArray_SimpleNew(2, nd, NPY_FLOAT64);
        if (!p) return -1;
        swap_ref(&self->pos, p);
        PyObject *v = PyArray_SimpleNew(2, nd, NPY_FLOAT64);
        if (!v) return -1;
        swap_ref(&self->vel, v);
        PyObject *m = PyArray_SimpleNew(1, nd, NPY_FLOAT64);
        if (!m) return -1;
        swap_ref(&self->mass, m);
        nd[1] = 8;
        PyObject *c = PyArray_SimpleNew(2, nd, NPY_INT32);
        if (!c) return -1;
        swap_ref(&self->connectivity, c);
        int rc;
        double *pp = (double *)PyArray_DATA((PyArrayObject *)p), *vp = (double *)PyArray_DATA((PyArrayObject *)v);
        double *mp = (double *)PyArray_DATA((PyArrayObject *)m);
        int *cp = (int *)PyArray_DATA((PyArrayObject *)c);
        Py_BEGIN_ALLOW_THREADS rc = strcmp(cloader, "gadget2") == 0 ? psib_load_gadget2(cfile, np, pp, vp, mp, cp)
                                                                   : psib_load_gevolution(cfile, np, pp, vp, mp, cp);
        Py_END_ALLOW_THREADS if (rc != PSIB_OK) {
            PyErr_Format(PyExc_ValueError, "Could not read %s: %s", cfile, psib_last_error());
            return -1;
        }
        self->block = 0;
        self->dim = 3;
        self->elemtype = 8;
        self->npart = np;
        self->nelem = np;
        self->periodic = 1;
        for (int i = 0; i < 3; ++i) {
            self->box[0][i] = 0.0;
            self->box[1][i] = boxsize;
        }
    } else {
        PyErr_SetString(PyExc_ValueError, "Invalid mesh loader.");
        return -1;
    }
    if (self->periodic) {
        PyObject *wb = Py_BuildValue("((ddd)(ddd))", self->box[0][0], self->box[0][1], self->box[0][2],
                                     self->box[1][0], self->box[1][1], self->box[1][2]);
        if (!wb) return -1;
        swap_ref(&self->wrapbox, wb);
    }
    return 0;
}

static PyObject *Mesh_new(PyTypeObject *type, PyObject *args, PyObject *kwds)
{
    (void)args;
    (void)kwds;
    Mesh *self = (Mesh *)type->tp_alloc(type, 0);
    if (!self) return NULL;
    PyObject **slots[5] = {&self->pos, &self->vel, &self->mass, &self->connectivity, &self->wrapbox};
    for (int i = 0; i < 5; ++i) {
        Py_INCREF(Py_None);
        *slots[i] = Py_None;
    }
    return (PyObject *)self;
}

static void Mesh_dealloc(Mesh *self)
{
    Py_XDECREF(self->pos);
    Py_XDECREF(self->vel);
    Py_XDECREF(self->mass);
    Py_XDECREF(self->connectivity);
    Py_XDECREF(self->wrapbox);
    Py_TYPE(self)->tp_free((PyObject *)self);
}

static PyMemberDef Mesh_members[] = {{"pos", T_OBJECT_EX, offsetof(Mesh, pos), 0, "pos"},
                                     {"vel", T_OBJECT_EX, offsetof(Mesh, vel), 0, "vel"},
                                     {"mass", T_OBJECT_EX, offsetof(Mesh, mass), 0, "mass"},
                                     {"connectivity", T_OBJECT_EX, offsetof(Mesh, connectivity), 0, "connectivity"},
                                     {"wrapbox", T_OBJECT_EX, offsetof(Mesh, wrapbox), 0, "wrapbox"},
                                     {NULL, 0, 0, 0, NULL}};

static PyTypeObject MeshType = {
    PyVarObject_HEAD_INIT(NULL, 0).tp_name = "PSI.Mesh",
    .tp_basicsize = sizeof(Mesh),
    .tp_dealloc = (destructor)Mesh_dealloc,
    .tp_flags = Py_TPFLAGS_DEFAULT | Py_TPFLAGS_BASETYPE,
    .tp_doc = "Mesh",
    .tp_members = Mesh_members,
    .tp_init = (initproc)Mesh_init,
    .tp_new = Mesh_new,
};

/* ------------------------------------------------------------ voxels() */

static PyObject *raise_status_of(const char *what, int rc)
{
    PyObject *exc = PyExc_RuntimeError;
    if (rc == PSIB_ERR_ARG) exc = PyExc_ValueError;
    else if (rc == PSIB_ERR_UNSUPPORTED) exc = PyExc_NotImplementedError;
    else if (rc == PSIB_ERR_NOMEM) exc = PyExc_MemoryError;
    PyErr_Format(exc, "%s failed (code %d): %s", what, rc, psib_last_error());
    return NULL;
}

static PyObject *raise_status(int rc) { return raise_status_of("PSI.voxels", rc); }

/* The library's view of a Mesh object's arrays. */
static void mesh_view(Mesh *mesh, psib_mesh *m)
{
    memset(m, 0, sizeof(*m));
    m->elemtype = mesh->elemtype;
    m->npart = mesh->npart;
    m->nelem = mesh->nelem;
    m->pos = (const double *)PyArray_DATA((PyArrayObject *)mesh->pos);
    m->vel = (const double *)PyArray_DATA((PyArrayObject *)mesh->vel);
    m->mass = (const double *)PyArray_DATA((PyArrayObject *)mesh->mass);
    if (mesh->block) {
        for (int i = 0; i < 3; ++i) m->block_dims[i] = mesh->nside[i];
    } else {
        m->connectivity = (const int *)PyArray_DATA((PyArrayObject *)mesh->connectivity);
    }
    m->periodic = mesh->periodic;
    memcpy(m->box, mesh->box, sizeof(m->box));
}

/* src/PSI.c:974-1018 */
static PyObject *PSI_voxels(PyObject *self, PyObject *args, PyObject *kwds)
{
    (void)self;
    Grid *grid;
    Mesh *mesh;
    char *modestr = "density", *precstr = "fp64", *critstr = "midpoint";
    double reftol = 1.0;
    int maxlvl = 0, det = 0;
    static char *kwlist[] = {"grid", "mesh", "mode", "refine_tolerance", "refine_max_lvl", "precision",
                             "deterministic", "refine_criterion", NULL};
    if (!PyArg_ParseTupleAndKeywords(args, kwds, "O!O!|sdispz", kwlist, &GridType, &grid, &MeshType, &mesh, &modestr,
                                     &reftol, &maxlvl, &precstr, &det, &critstr))
        return NULL;
    int crit;
    if (!critstr || strcmp(critstr, "midpoint") == 0) crit = PSIB_REFINE_MIDPOINT;
    else if (strcmp(critstr, "stretch") == 0) crit = PSIB_REFINE_STRETCH;
    else {
        PyErr_Format(PyExc_ValueError, "Invalid refine_criterion for PSI.voxels(): %s", critstr);
        return NULL;
    }
    if (grid->ctype != GRID_CART) {
        PyErr_SetString(PyExc_ValueError, "Only cartesian grids are supported by PSI.voxels()");
        return NULL;
    }
    if (mesh->dim != grid->dim) {
        PyErr_SetString(PyExc_ValueError, "Input mesh and grid must have the same number of dimensions");
        return NULL;
    }
    int mode;
    if (strcmp(modestr, "density") == 0) mode = PSIB_MODE_DENSITY;
    else if (strcmp(modestr, "annihilation") == 0) mode = PSIB_MODE_ANNIHILATION;
    else {
        PyErr_Format(PyExc_ValueError, "Invalid mode for PSI.voxels(): %s", modestr);
        return NULL;
    }
    int prec;
    if (strcmp(precstr, "fp64") == 0) prec = PSIB_FP64;
    else if (strcmp(precstr, "mixed") == 0) prec = PSIB_MIXED;
    else if (strcmp(precstr, "fp64-central") == 0) prec = PSIB_FP64_CENTRAL;
    else {
        PyErr_Format(PyExc_ValueError, "Invalid precision for PSI.voxels(): %s", precstr);
        return NULL;
    }
    psib_grid g;
    memset(&g, 0, sizeof(g));
    for (int i = 0; i < 3; ++i) {
        g.n[i] = grid->cn[i];
        g.window[0][i] = grid->window[0][i];
        g.window[1][i] = grid->window[1][i];
        g.d[i] = grid->cd[i];
    }
    /* the field dict may have been edited; bind the arrays it holds now */
    static const char *names[6] = {"m", "x", "v", "xx", "xv", "vv"};
    static const int comps[6] = {1, 3, 3, 9, 9, 9};
    for (int f = 0; f < 6; ++f) {
        if (!grid->cfields[f]) continue;
        PyObject *a = PyDict_GetItemString(grid->fields, names[f]);
        npy_intp want = (npy_intp)grid->cn[0] * grid->cn[1] * grid->cn[2] * comps[f];
        if (!a || !PyArray_Check(a) || PyArray_TYPE((PyArrayObject *)a) != NPY_FLOAT64 ||
            !PyArray_IS_C_CONTIGUOUS((PyArrayObject *)a) || !PyArray_ISWRITEABLE((PyArrayObject *)a) ||
            PyArray_SIZE((PyArrayObject *)a) != want) {
            PyErr_Format(PyExc_ValueError, "grid field '%s' must stay a writable C-contiguous float64 array", names[f]);
            return NULL;
        }
        g.fields[f] = (double *)PyArray_DATA((PyArrayObject *)a);
    }
    psib_mesh m;
    mesh_view(mesh, &m);

    psib_options o;
    memset(&o, 0, sizeof(o));
    o.precision = prec;
    o.refine_mode = crit;
    o.deterministic = det;
    o.memory = PSIB_HOST;
    o.device = -1;
    psib_stats stats;
    o.stats = &stats;
    int rc;
    Py_BEGIN_ALLOW_THREADS rc = psib_voxels(&g, &m, mode, reftol, maxlvl, &o);
    Py_END_ALLOW_THREADS if (rc != PSIB_OK) return raise_status(rc);
    g_last_stats = stats;
    Py_RETURN_NONE;
}

static PyObject *PSI_last_stats(PyObject *self, PyObject *noargs)
{
    (void)self;
    (void)noargs;
    const psib_stats *s = &g_last_stats;
    return Py_BuildValue("{s:L,s:L,s:L,s:L,s:L,s:L,s:i,s:i,s:f,s:f,s:f,s:f,s:L,s:L,s:L,s:L,s:i}", "elements_kept",
                         s->elements_kept, "tets", s->tets, "tet_images", s->tet_images, "fragments", s->fragments,
                         "frag_verts", s->frag_verts, "splits", s->splits, "passes", s->passes, "chunks", s->chunks,
                         "ms_total", (double)s->ms_total, "ms_clip", (double)s->ms_clip, "ms_tess", (double)s->ms_tess,
                         "ms_final", (double)s->ms_final, "clip_launches", s->clip_launches, "kernel_launches",
                         s->kernel_launches, "walk_bytes", s->walk_bytes, "corrected_items", s->corrected_items,
                         "accumulation", s->accumulation);
}

static PyObject *PSI_device_count(PyObject *self, PyObject *noargs)
{
    (void)self;
    (void)noargs;
    return PyLong_FromLong(psib_device_count());
}

/* ------------------------------------------------------------ RStarTree */

/* PSI.RStarTree(mesh, initial_capacity=1024) (src/PSI.c:809-962): the spatial
 * index of the mesh's elements.  It keeps the mesh and the cull window of the
 * reference's tree (the periodic box of a periodic mesh, +-1e30 for an open
 * one, src/PSI.c:877-893); its first query builds the library's device index
 * (psib_index_create: the mesh, its element boxes and a cell grid over them, as
 * the mesh is at that moment), which later queries and PSI.VDF(..., tree)
 * reuse. */
typedef struct {
    PyObject_HEAD PyObject *mesh;
    double window[2][3];
    psib_index *ix;
} RStarTree;

static int RStarTree_init(RStarTree *self, PyObject *args, PyObject *kwds)
{
    Mesh *mesh = NULL;
    int init_cap = 1024;
    static char *kwlist[] = {"mesh", "initial_capacity", NULL};
    if (!PyArg_ParseTupleAndKeywords(args, kwds, "O!|i", kwlist, &MeshType, &mesh, &init_cap)) return -1;
    (void)init_cap;
    for (int i = 0; i < 3; ++i) {
        self->window[0][i] = mesh->periodic ? mesh->box[0][i] : -1.0e30;
        self->window[1][i] = mesh->periodic ? mesh->box[1][i] : 1.0e30;
    }
    if (self->ix) {
        psib_index_destroy(self->ix);
        self->ix = NULL;
    }
    Py_INCREF(mesh);
    swap_ref(&self->mesh, (PyObject *)mesh);
    return 0;
}

static PyObject *RStarTree_new(PyTypeObject *type, PyObject *args, PyObject *kwds)
{
    (void)args;
    (void)kwds;
    RStarTree *self = (RStarTree *)type->tp_alloc(type, 0);
    return (PyObject *)self;
}

static void RStarTree_dealloc(RStarTree *self)
{
    if (self->ix) psib_index_destroy(self->ix);
    Py_XDECREF(self->mesh);
    Py_TYPE(self)->tp_free((PyObject *)self);
}

/* The tree's device index, built on first use (0, or -1 with an exception set). */
static int tree_index(RStarTree *self, const char *what)
{
    if (self->ix) return 0;
    if (!self->mesh) {
        PyErr_SetString(PyExc_ValueError, "RStarTree has no mesh");
        return -1;
    }
    psib_mesh m;
    mesh_view((Mesh *)self->mesh, &m);
    psib_index *ix = NULL;
    int rc;
    Py_BEGIN_ALLOW_THREADS rc = psib_index_create(&m, (const double(*)[3])self->window, &ix, NULL);
    Py_END_ALLOW_THREADS if (rc != PSIB_OK)
    {
        raise_status_of(what, rc);
        return -1;
    }
    self->ix = ix;
    return 0;
}

/* A float64 / int32 array of the first n entries of `a` (which holds at least n). */
static PyObject *head_of(PyObject *a, npy_intp n)
{
    PyArrayObject *arr = (PyArrayObject *)a;
    const int nd = PyArray_NDIM(arr);
    npy_intp dims[2] = {n, nd > 1 ? PyArray_DIMS(arr)[1] : 0};
    PyObject *out = PyArray_SimpleNew(nd, dims, PyArray_TYPE(arr));
    if (!out) return NULL;
    const size_t row = (size_t)PyArray_ITEMSIZE(arr) * (nd > 1 ? (size_t)dims[1] : 1);
    if (n > 0) memcpy(PyArray_DATA((PyArrayObject *)out), PyArray_DATA(arr), (size_t)n * row);
    return out;
}

/* src/PSI.c:817-862: int32 indices of the elements whose box touches `box` */
static PyObject *RStarTree_query(RStarTree *self, PyObject *args, PyObject *kwds)
{
    PyObject *box;
    double q[6];
    static char *kwlist[] = {"box", NULL};
    if (!PyArg_ParseTupleAndKeywords(args, kwds, "O", kwlist, &box)) return NULL;
    if (!PyArg_ParseTuple(box, "(ddd)(ddd)", &q[0], &q[1], &q[2], &q[3], &q[4], &q[5])) {
        PyErr_SetString(PyExc_TypeError, "Query box must be a tuple containing two tuples of 3 values each");
        return NULL;
    }
    if (tree_index(self, "PSI.RStarTree.query") < 0) return NULL;
    long long off[2] = {0, 0};
    npy_intp cap = 1024;
    for (int attempt = 0; attempt < 2; ++attempt) {
        PyObject *out = PyArray_SimpleNew(1, &cap, NPY_INT32);
        if (!out) return NULL;
        int *dst = (int *)PyArray_DATA((PyArrayObject *)out);
        int rc;
        Py_BEGIN_ALLOW_THREADS rc = psib_index_query(self->ix, q, 1, off, dst, (long long)cap, NULL);
        Py_END_ALLOW_THREADS if (rc == PSIB_ERR_OVERFLOW && attempt == 0)
        {
            Py_DECREF(out);
            cap = (npy_intp)off[1];
            continue;
        }
        if (rc != PSIB_OK) {
            Py_DECREF(out);
            return raise_status_of("PSI.RStarTree.query", rc);
        }
        PyObject *res = head_of(out, (npy_intp)off[1]);
        Py_DECREF(out);
        return res;
    }
    PyErr_SetString(PyExc_RuntimeError, "PSI.RStarTree.query: the result size changed between calls");
    return NULL;
}

static PyMemberDef RStarTree_members[] = {{"mesh", T_OBJECT_EX, offsetof(RStarTree, mesh), READONLY, "mesh"},
                                          {NULL, 0, 0, 0, NULL}};

static PyMethodDef RStarTree_methods[] = {
    {"query", (PyCFunction)(void (*)(void))RStarTree_query, METH_VARARGS | METH_KEYWORDS, "Query the RStarTree."},
    {NULL, NULL, 0, NULL}};

static PyTypeObject RStarTreeType = {
    PyVarObject_HEAD_INIT(NULL, 0).tp_name = "PSI.RStarTree",
    .tp_basicsize = sizeof(RStarTree),
    .tp_dealloc = (destructor)RStarTree_dealloc,
    .tp_flags = Py_TPFLAGS_DEFAULT | Py_TPFLAGS_BASETYPE,
    .tp_doc = "RStarTree",
    .tp_methods = RStarTree_methods,
    .tp_members = RStarTree_members,
    .tp_init = (initproc)RStarTree_init,
    .tp_new = RStarTree_new,
};

/* ------------------------------------------------------------ VDF */

/* PSI.VDF(mesh, sample_pos, tree=None, refine_tolerance=1.0, refine_max_lvl=0)
 * (src/PSI.c:1022-1057): (rho, vel) of every stream at sample_pos.  Without a
 * tree the elements are culled against the mesh's box, as the reference's own
 * tree for this call is (src/cpsi.c:206-209); with one, the tree's index (and
 * so its window) is used. */
static PyObject *PSI_VDF(PyObject *self, PyObject *args, PyObject *kwds)
{
    (void)self;
    Mesh *mesh = NULL;
    RStarTree *tree = NULL;
    double s[3], reftol = 1.0;
    int maxlvl = 0;
    static char *kwlist[] = {"mesh", "sample_pos", "tree", "refine_tolerance", "refine_max_lvl", NULL};
    if (!PyArg_ParseTupleAndKeywords(args, kwds, "O!(ddd)|O!di", kwlist, &MeshType, &mesh, &s[0], &s[1], &s[2],
                                     &RStarTreeType, &tree, &reftol, &maxlvl))
        return NULL;
    if (tree && tree_index(tree, "PSI.VDF") < 0) return NULL;
    psib_mesh m;
    mesh_view(mesh, &m);
    double win[2][3];
    memcpy(win, mesh->box, sizeof(win));
    long long off[2] = {0, 0};
    npy_intp cap = 256;
    for (int attempt = 0; attempt < 2; ++attempt) {
        npy_intp nd[2] = {cap, 3};
        PyObject *rho = PyArray_SimpleNew(1, nd, NPY_FLOAT64);
        PyObject *vel = PyArray_SimpleNew(2, nd, NPY_FLOAT64);
        if (!rho || !vel) {
            Py_XDECREF(rho);
            Py_XDECREF(vel);
            return NULL;
        }
        double *r = (double *)PyArray_DATA((PyArrayObject *)rho), *v = (double *)PyArray_DATA((PyArrayObject *)vel);
        int rc;
        Py_BEGIN_ALLOW_THREADS if (tree) rc =
            psib_index_sample_vdf(tree->ix, s, 1, reftol, maxlvl, off, r, v, (long long)cap, NULL);
        else rc = psib_sample_vdf(&m, (const double(*)[3])win, s, 1, reftol, maxlvl, off, r, v, (long long)cap, NULL);
        Py_END_ALLOW_THREADS if (rc == PSIB_ERR_OVERFLOW && attempt == 0)
        {
            Py_DECREF(rho);
            Py_DECREF(vel);
            cap = (npy_intp)off[1];
            continue;
        }
        if (rc != PSIB_OK) {
            Py_DECREF(rho);
            Py_DECREF(vel);
            return raise_status_of("PSI.VDF", rc);
        }
        PyObject *rh = head_of(rho, (npy_intp)off[1]), *vh = head_of(vel, (npy_intp)off[1]);
        Py_DECREF(rho);
        Py_DECREF(vel);
        if (!rh || !vh) {
            Py_XDECREF(rh);
            Py_XDECREF(vh);
            return NULL;
        }
        PyObject *ret = Py_BuildValue("OO", rh, vh);
        Py_DECREF(rh);
        Py_DECREF(vh);
        return ret;
    }
    PyErr_SetString(PyExc_RuntimeError, "PSI.VDF: the result size changed between calls");
    return NULL;
}

static PyMethodDef module_methods[] = {
    {"voxels", (PyCFunction)(void (*)(void))PSI_voxels, METH_VARARGS | METH_KEYWORDS, "Voxelizes"},
    {"VDF", (PyCFunction)(void (*)(void))PSI_VDF, METH_VARARGS | METH_KEYWORDS, "VDF"},
    {"last_stats", PSI_last_stats, METH_NOARGS, "Work counters and device timings of the last voxels() call"},
    {"device_count", PSI_device_count, METH_NOARGS, "Number of visible CUDA devices"},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef PSImodule = {PyModuleDef_HEAD_INIT, "PSI", "PSI, the phase space intersector (B200)", -1,
                                       module_methods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit_PSI(void)
{
    PyObject *m = PyModule_Create(&PSImodule);
    if (!m) return NULL;
    import_array();
    if (PyType_Ready(&MeshType) < 0 || PyType_Ready(&GridType) < 0 || PyType_Ready(&RStarTreeType) < 0) return NULL;
    Py_INCREF(&MeshType);
    PyModule_AddObject(m, "Mesh", (PyObject *)&MeshType);
    Py_INCREF(&RStarTreeType);
    PyModule_AddObject(m, "RStarTree", (PyObject *)&RStarTreeType);
    Py_INCREF(&GridType);
    PyModule_AddObject(m, "Grid", (PyObject *)&GridType);
    return m;
}
