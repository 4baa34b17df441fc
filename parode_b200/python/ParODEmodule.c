/*
 * ParODEmodule.c -- Python 3 extension module `ParODE` over libParODEShared.so.
 *
 * Same module name, function names, argument lists and return tuples as the
 * reference's Python 2 module (PythonInterface/ParODEmodule.c:450-474), so
 * scripts such as PythonInterface/TestPythonODESolvers.py run unchanged apart
 * from their Python 2 print statements.  Differences: the module is silent
 * (the reference echoes every SimulateODE argument to stdout), any sequence
 * is accepted where the reference demanded a list, and invalid matrices
 * return None with a proper reference count.
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>

#include <stdlib.h>

#include <ParODECInterface.h>

static PyObject* ParODEError;

/* Reference ParODEmodule.c:7-16. */
static PyObject* py_GetErrorDescription(PyObject* self, PyObject* args)
{
    int code;
    char text[256];
    if (!PyArg_ParseTuple(args, "i", &code)) return NULL;
    GetErrorDescription(&code, text);
    return Py_BuildValue("s", text);
}

/* Reference ParODEmodule.c:19-42 (kernel folders are not needed). */
static PyObject* py_InitializeAllGPUs(PyObject* self, PyObject* args)
{
    int err = 0;
    char empty[1] = {0};
    InitializeAllGPUs(empty, empty, &err);
    return Py_BuildValue("i", err);
}

/* Reference ParODEmodule.c:45-75. */
static PyObject* py_GetAvailableGPUs(PyObject* self, PyObject* args)
{
    int n = 0, err = 0, ids[64];
    GetAvailableGPUs(&n, ids, &err);
    PyObject* lst = PyList_New(n);
    if (!lst) return NULL;
    for (int i = 0; i < n; ++i) PyList_SET_ITEM(lst, i, PyLong_FromLong(ids[i]));
    return Py_BuildValue("(Ni)", lst, err);
}

/* Reference ParODEmodule.c:78-87. */
static PyObject* py_GetDeviceName(PyObject* self, PyObject* args)
{
    int id, err = 0;
    char name[256];
    if (!PyArg_ParseTuple(args, "i", &id)) return NULL;
    name[0] = 0;
    GetDeviceName(&id, name, &err);
    return Py_BuildValue("(si)", name, err);
}

/* Reference ParODEmodule.c:90-133. */
static PyObject* py_InitializeSelectedGPUs(PyObject* self, PyObject* args)
{
    PyObject* obj;
    if (!PyArg_ParseTuple(args, "O", &obj)) return NULL;
    PyObject* seq = PySequence_Fast(obj, "InitializeSelectedGPUs expects a list of device ids");
    if (!seq) return NULL;
    Py_ssize_t n = PySequence_Fast_GET_SIZE(seq);
    int* ids = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!ids) {
        Py_DECREF(seq);
        return PyErr_NoMemory();
    }
    for (Py_ssize_t i = 0; i < n; ++i) {
        long v = PyLong_AsLong(PySequence_Fast_GET_ITEM(seq, i));
        if (v == -1 && PyErr_Occurred()) {
            free(ids);
            Py_DECREF(seq);
            return NULL;
        }
        ids[i] = (int)v;
    }
    Py_DECREF(seq);
    int cnt = (int)n, err = 0;
    char empty[1] = {0};
    InitializeSelectedGPUs(&cnt, ids, empty, empty, &err);
    free(ids);
    return Py_BuildValue("i", err);
}

/* Row-major float copy of a list of rows; an empty list is an absent
 * matrix.  Returns 0 (with or without a Python error set) on malformed input
 * (reference DisassembleMatrix, ParODEmodule.c:135-183). */
static int to_matrix(PyObject* obj, float** out, int* rows, int* cols)
{
    *out = NULL;
    *rows = *cols = 0;
    PyObject* seq = PySequence_Fast(obj, "matrix must be a list of rows");
    if (!seq) return 0;
    Py_ssize_t r = PySequence_Fast_GET_SIZE(seq);
    if (r == 0) {
        Py_DECREF(seq);
        return 1;
    }
    int ok = 1;
    Py_ssize_t c = -1;
    float* m = NULL;
    for (Py_ssize_t i = 0; i < r && ok; ++i) {
        PyObject* row = PySequence_Fast(PySequence_Fast_GET_ITEM(seq, i), "matrix rows must be lists");
        if (!row) {
            ok = 0;
            break;
        }
        Py_ssize_t rc = PySequence_Fast_GET_SIZE(row);
        if (c < 0) {
            c = rc;
            m = (float*)malloc(sizeof(float) * (size_t)(r * (c > 0 ? c : 1)));
            if (!m) ok = 0;
        } else if (rc != c) {
            ok = 0;
        }
        for (Py_ssize_t j = 0; ok && j < rc; ++j) {
            double v = PyFloat_AsDouble(PySequence_Fast_GET_ITEM(row, j));
            if (v == -1.0 && PyErr_Occurred()) ok = 0;
            else m[i * c + j] = (float)v;
        }
        Py_DECREF(row);
    }
    Py_DECREF(seq);
    if (!ok) {
        free(m);
        return 0;
    }
    if (c == 0) {
        free(m);
        m = NULL;
        r = 0;
    }
    *out = m;
    *rows = (int)r;
    *cols = (int)(c > 0 ? c : 0);
    return 1;
}

/* Reference ParODEmodule.c:219-409: SimulateODE(A, B, C, D, uIndex, tStart,
 * tStep, nSteps, x0, solver) -> (tList, [[y_0..y_p-1] per step], nErr). */
static PyObject* py_SimulateODE(PyObject* self, PyObject* args)
{
    PyObject *Ao, *Bo, *Co, *Do, *xo;
    int uIndex, nSteps, solver;
    double tStart, tStep;
    if (!PyArg_ParseTuple(args, "OOOOiddiOi", &Ao, &Bo, &Co, &Do, &uIndex, &tStart, &tStep, &nSteps, &xo, &solver))
        return NULL;
    float *A = NULL, *B = NULL, *C = NULL, *D = NULL, *x0 = NULL, *tv = NULL, *yv = NULL;
    int r, c, nStates = 0, nInputs = 0, nOutputs = 0, zB = 0, zC = 0, zD = 0;
    PyObject* result = NULL;
    if (!to_matrix(Ao, &A, &r, &c) || r == 0 || r != c) goto invalid;
    nStates = r;
    if (!to_matrix(Bo, &B, &r, &c)) goto invalid;
    if (r == 0) zB = 1;
    else if (r == nStates) nInputs = c;
    else goto invalid;
    if (!to_matrix(Co, &C, &r, &c)) goto invalid;
    if (r == 0) zC = 1;
    else if (c == nStates) nOutputs = r;
    else goto invalid;
    if (!to_matrix(Do, &D, &r, &c)) goto invalid;
    if (r == 0) {
        zD = 1;
    } else {
        if (zB) nInputs = c;
        if (zC) nOutputs = r;
        if (nInputs != c || nOutputs != r) goto invalid;
    }
    if (zC && zD) nOutputs = nStates;
    {
        PyObject* seq = PySequence_Fast(xo, "x0 must be a list");
        if (!seq) goto invalid;
        if (PySequence_Fast_GET_SIZE(seq) != nStates) {
            Py_DECREF(seq);
            goto invalid;
        }
        x0 = (float*)malloc(sizeof(float) * (size_t)nStates);
        for (int i = 0; x0 && i < nStates; ++i) {
            double v = PyFloat_AsDouble(PySequence_Fast_GET_ITEM(seq, i));
            if (v == -1.0 && PyErr_Occurred()) {
                Py_DECREF(seq);
                goto invalid;
            }
            x0[i] = (float)v;
        }
        Py_DECREF(seq);
        if (!x0) goto invalid;
    }
    {
        double tEnd = tStart + (nSteps - 1) * tStep;
        int nOut = 0, err = 0;
        int cap = nSteps > 0 ? nSteps : 1;
        tv = (float*)malloc(sizeof(float) * (size_t)cap);
        yv = (float*)malloc(sizeof(float) * (size_t)cap * (size_t)nOutputs);
        if (!tv || !yv) {
            PyErr_NoMemory();
            goto fail;
        }
        Py_BEGIN_ALLOW_THREADS
        SimulateODE(A, B, C, D, &nInputs, &nStates, &nOutputs, &zB, &zC, &zD, &uIndex, &tStart, &tEnd, &tStep, x0,
                    &solver, tv, yv, &nOut, &err);
        Py_END_ALLOW_THREADS
        if (err != 0 || nOut > cap) nOut = 0;
        PyObject* tl = PyList_New(nOut);
        PyObject* xl = PyList_New(nOut);
        if (!tl || !xl) {
            Py_XDECREF(tl);
            Py_XDECREF(xl);
            goto fail;
        }
        for (int k = 0; k < nOut; ++k) {
            PyList_SET_ITEM(tl, k, PyFloat_FromDouble(tv[k]));
            PyObject* row = PyList_New(nOutputs);
            for (int o = 0; row && o < nOutputs; ++o)
                PyList_SET_ITEM(row, o, PyFloat_FromDouble(yv[(size_t)k * nOutputs + o]));
            PyList_SET_ITEM(xl, k, row);
        }
        result = Py_BuildValue("(NNi)", tl, xl, err);
    }
    goto fail;
invalid:
    PyErr_Clear();
    Py_INCREF(Py_None);
    result = Py_None;
fail:
    free(A);
    free(B);
    free(C);
    free(D);
    free(x0);
    free(tv);
    free(yv);
    return result;
}

/* Reference ParODEmodule.c:412-421. */
static PyObject* py_RegisterInput(PyObject* self, PyObject* args)
{
    char* src;
    if (!PyArg_ParseTuple(args, "s", &src)) return NULL;
    int idx = 0, err = 0;
    RegisterInput(src, &idx, &err);
    return Py_BuildValue("(ii)", idx, err);
}

/* Reference ParODEmodule.c:425-430. */
static PyObject* py_CloseGPU(PyObject* self, PyObject* args)
{
    CloseGPUC();
    Py_RETURN_NONE;
}

/* Reference ParODEmodule.c:433-448. */
static PyObject* py_StartTimer(PyObject* self, PyObject* args)
{
    int err = 0;
    StartTimer(&err);
    return Py_BuildValue("i", err);
}

static PyObject* py_StopTimer(PyObject* self, PyObject* args)
{
    float ms = 0.0f;
    int err = 0;
    StopTimer(&ms, &err);
    return Py_BuildValue("(fi)", ms, err);
}

static PyMethodDef kMethods[] = {
    {"GetErrorDescription", py_GetErrorDescription, METH_VARARGS, "Get Error Description String."},
    {"InitializeAllGPUs", py_InitializeAllGPUs, METH_VARARGS, "Initialize all available GPUs."},
    {"GetAvailableGPUs", py_GetAvailableGPUs, METH_VARARGS, "Retrieve all the available GPUs."},
    {"GetDeviceName", py_GetDeviceName, METH_VARARGS, "Get the device name."},
    {"InitializeSelectedGPUs", py_InitializeSelectedGPUs, METH_VARARGS, "Initialize Selected GPUs."},
    {"SimulateODE", py_SimulateODE, METH_VARARGS, "Simulate an LTI system."},
    {"RegisterInput", py_RegisterInput, METH_VARARGS, "Register an input kernel."},
    {"CloseGPU", py_CloseGPU, METH_VARARGS, "Release GPU resources."},
    {"StartTimer", py_StartTimer, METH_VARARGS, "Start GPU timer."},
    {"StopTimer", py_StopTimer, METH_VARARGS, "Retrieve timer value."},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef kModule = {PyModuleDef_HEAD_INIT, "ParODE",
                                     "GPU-accelerated LTI simulation (B200 build of ParODE).", -1, kMethods};

PyMODINIT_FUNC PyInit_ParODE(void)
{
    PyObject* m = PyModule_Create(&kModule);
    if (!m) return NULL;
    ParODEError = PyErr_NewException("ParODE.error", NULL, NULL);
    Py_XINCREF(ParODEError);
    if (PyModule_AddObject(m, "error", ParODEError) < 0) {
        Py_XDECREF(ParODEError);
        Py_CLEAR(ParODEError);
        Py_DECREF(m);
        return NULL;
    }
    return m;
}
