// MEX runtime stand-in: mxArray, mxGPUArray and the mex* calls, in C++.
//
// TEST INFRASTRUCTURE ONLY (see matrix.h).  It lets two kinds of MEX code
// run without MATLAB:
//   * the reference's own kernels, Runtime/solver/decompBlockLU.cu and
//     Runtime/solver/applyBlockLU.cu, compiled unchanged from their sources
//     (the oracle's pin for the complex-single block LU, and the reference's
//     GPU path timed on the same device);
//   * this repository's gateways in waveforminversionust_b200/mex/, to test
//     the drop-in boundary end to end.
// A host drives a MEX function through the mexshim_* entry points below:
// it builds input mxArrays (wrapping existing device memory for gpuArrays),
// calls mexFunction through mexshim_call, which catches the exception that
// mexErrMsgIdAndTxt raises, and reads the outputs.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gpu/mxGPUArray.h"
#include "mex.h"

namespace {

struct Buffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    bool device = false;
    bool owned = true;
    ~Buffer() {
        if (!owned || !ptr) return;
        if (device) {
            cudaFree(ptr);
            live_device_bytes(-(long long)bytes);
        } else {
            std::free(ptr);
        }
    }
    static long long live_device_bytes(long long delta) {
        static std::mutex m;
        static long long live = 0;
        std::lock_guard<std::mutex> g(m);
        live += delta;
        return live;
    }
};

struct MexError : std::runtime_error {
    std::string id;
    MexError(const std::string &i, const std::string &msg) : std::runtime_error(msg), id(i) {}
};

size_t element_bytes(mxClassID c) {
    switch (c) {
        case mxLOGICAL_CLASS: case mxCHAR_CLASS: case mxINT8_CLASS: case mxUINT8_CLASS: return 1;
        case mxINT16_CLASS: case mxUINT16_CLASS: return 2;
        case mxINT32_CLASS: case mxUINT32_CLASS: case mxSINGLE_CLASS: return 4;
        case mxINT64_CLASS: case mxUINT64_CLASS: case mxDOUBLE_CLASS: return 8;
        default: return 0;
    }
}

size_t count(const std::vector<size_t> &d) {
    size_t n = 1;
    for (size_t v : d) n *= v;
    return n;
}

std::vector<size_t> normalise(size_t nd, const size_t *dims) {
    std::vector<size_t> d(dims, dims + nd);
    while (d.size() < 2) d.push_back(1);
    while (d.size() > 2 && d.back() == 1) d.pop_back();      // trailing singleton dimensions, as MATLAB drops them
    return d;
}

std::shared_ptr<Buffer> device_buffer(size_t bytes, bool zero) {
    auto b = std::make_shared<Buffer>();
    b->device = true;
    b->bytes = bytes;
    if (bytes) {
        if (cudaMalloc(&b->ptr, bytes) != cudaSuccess) {
            cudaGetLastError();
            throw MexError("parallel:gpu:array:OOM", "Out of memory on device");
        }
        Buffer::live_device_bytes((long long)bytes);
        if (zero) cudaMemset(b->ptr, 0, bytes);
    }
    return b;
}

std::shared_ptr<Buffer> host_buffer(size_t bytes) {
    auto b = std::make_shared<Buffer>();
    b->bytes = bytes;
    b->ptr = std::calloc(bytes ? bytes : 1, 1);
    return b;
}

std::vector<void (*)(void)> &exit_hooks() {
    static std::vector<void (*)(void)> h;
    return h;
}

}  // namespace

struct mxArray_tag {
    enum Kind { NUMERIC, STRUCT, CHAR } kind = NUMERIC;
    bool gpu = false;
    mxClassID cls = mxDOUBLE_CLASS;
    mxComplexity cplx = mxREAL;
    std::vector<size_t> dims{0, 0};
    std::shared_ptr<Buffer> data;
    std::vector<std::string> names;     // 1 x 1 struct
    std::vector<mxArray *> values;
    std::string text;
    ~mxArray_tag() {
        for (mxArray *v : values) delete v;
    }
    size_t bytes() const { return count(dims) * element_bytes(cls) * (cplx == mxCOMPLEX ? 2 : 1); }
};

struct mxGPUArray_tag {
    mxClassID cls = mxSINGLE_CLASS;
    mxComplexity cplx = mxREAL;
    std::vector<size_t> dims;
    std::shared_ptr<Buffer> data;
};

namespace {

mxArray *numeric(std::vector<size_t> dims, mxClassID cls, mxComplexity cplx) {
    auto *a = new mxArray;
    a->cls = cls;
    a->cplx = cplx;
    a->dims = std::move(dims);
    a->data = host_buffer(a->bytes());
    return a;
}

void require_host(const mxArray *a, const char *what) {
    if (!a) throw MexError("MATLAB:mexshim:null", std::string(what) + ": null mxArray");
    if (a->gpu) throw MexError("MATLAB:mexshim:gpu", std::string(what) + ": the data of a gpuArray is not host memory");
}

}  // namespace

extern "C" {

void *mxMalloc(size_t n) { return std::malloc(n ? n : 1); }
void *mxCalloc(size_t n, size_t size) { return std::calloc(n ? n : 1, size ? size : 1); }
void mxFree(void *p) { std::free(p); }

mxArray *mxCreateDoubleScalar(double v) {
    mxArray *a = numeric({1, 1}, mxDOUBLE_CLASS, mxREAL);
    *(double *)a->data->ptr = v;
    return a;
}

mxArray *mxCreateLogicalScalar(bool v) {
    mxArray *a = numeric({1, 1}, mxLOGICAL_CLASS, mxREAL);
    *(mxLogical *)a->data->ptr = v;
    return a;
}

mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID cls, mxComplexity cplx) {
    return numeric(normalise(ndim, dims), cls, cplx);
}

mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity cplx) {
    return numeric({m, n}, cls, cplx);
}

mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity cplx) { return numeric({m, n}, mxDOUBLE_CLASS, cplx); }

mxArray *mxCreateString(const char *s) {
    auto *a = new mxArray;
    a->kind = mxArray::CHAR;
    a->cls = mxCHAR_CLASS;
    a->text = s ? s : "";
    a->dims = {1, a->text.size()};
    return a;
}

mxArray *mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char **names) {
    if (m != 1 || n != 1) throw MexError("MATLAB:mexshim:struct", "only 1 x 1 structs are supported");
    auto *a = new mxArray;
    a->kind = mxArray::STRUCT;
    a->cls = mxSTRUCT_CLASS;
    a->dims = {1, 1};
    for (int i = 0; i < nfields; ++i) {
        a->names.push_back(names[i]);
        a->values.push_back(nullptr);
    }
    return a;
}

void mxDestroyArray(mxArray *a) { delete a; }

void mxSetField(mxArray *s, mwIndex index, const char *name, mxArray *value) {
    if (!s || s->kind != mxArray::STRUCT || index != 0) throw MexError("MATLAB:mexshim:struct", "bad struct field set");
    for (size_t i = 0; i < s->names.size(); ++i)
        if (s->names[i] == name) {
            delete s->values[i];
            s->values[i] = value;
            return;
        }
    throw MexError("MATLAB:mexshim:struct", std::string("no field ") + name);
}

mxArray *mxGetField(const mxArray *s, mwIndex index, const char *name) {
    if (!s || s->kind != mxArray::STRUCT || index != 0) return nullptr;
    for (size_t i = 0; i < s->names.size(); ++i)
        if (s->names[i] == name) return s->values[i];
    return nullptr;
}

mxClassID mxGetClassID(const mxArray *a) { return a ? a->cls : mxUNKNOWN_CLASS; }
bool mxIsDouble(const mxArray *a) { return a && a->cls == mxDOUBLE_CLASS; }
bool mxIsSingle(const mxArray *a) { return a && a->cls == mxSINGLE_CLASS; }
bool mxIsComplex(const mxArray *a) { return a && a->cplx == mxCOMPLEX; }
bool mxIsChar(const mxArray *a) { return a && a->kind == mxArray::CHAR; }
bool mxIsStruct(const mxArray *a) { return a && a->kind == mxArray::STRUCT; }
bool mxIsLogical(const mxArray *a) { return a && a->cls == mxLOGICAL_CLASS; }
bool mxIsNumeric(const mxArray *a) {
    return a && a->kind == mxArray::NUMERIC && a->cls != mxLOGICAL_CLASS && a->cls != mxCHAR_CLASS;
}
bool mxIsInt32(const mxArray *a) { return a && a->cls == mxINT32_CLASS; }
bool mxIsUint8(const mxArray *a) { return a && a->cls == mxUINT8_CLASS; }
bool mxIsUint64(const mxArray *a) { return a && a->cls == mxUINT64_CLASS; }
bool mxIsEmpty(const mxArray *a) { return !a || count(a->dims) == 0; }
bool mxIsLogicalScalar(const mxArray *a) {
    return a && !a->gpu && a->cls == mxLOGICAL_CLASS && count(a->dims) == 1;
}
bool mxIsLogicalScalarTrue(const mxArray *a) {
    return mxIsLogicalScalar(a) && *(const mxLogical *)a->data->ptr;
}

mwSize mxGetNumberOfDimensions(const mxArray *a) { return a ? a->dims.size() : 0; }
const mwSize *mxGetDimensions(const mxArray *a) { return a ? a->dims.data() : nullptr; }
size_t mxGetNumberOfElements(const mxArray *a) { return a ? count(a->dims) : 0; }
size_t mxGetM(const mxArray *a) { return a ? a->dims[0] : 0; }
size_t mxGetN(const mxArray *a) { return a ? count(a->dims) / (a->dims[0] ? a->dims[0] : 1) : 0; }

void *mxGetData(const mxArray *a) {
    require_host(a, "mxGetData");
    return a->data ? a->data->ptr : nullptr;
}
double *mxGetDoubles(const mxArray *a) { return mxIsDouble(a) && !a->gpu ? (double *)a->data->ptr : nullptr; }
float *mxGetSingles(const mxArray *a) { return mxIsSingle(a) && !a->gpu ? (float *)a->data->ptr : nullptr; }
int32_t *mxGetInt32s(const mxArray *a) { return mxIsInt32(a) && !a->gpu ? (int32_t *)a->data->ptr : nullptr; }
uint8_t *mxGetUint8s(const mxArray *a) { return mxIsUint8(a) && !a->gpu ? (uint8_t *)a->data->ptr : nullptr; }
uint64_t *mxGetUint64s(const mxArray *a) { return mxIsUint64(a) && !a->gpu ? (uint64_t *)a->data->ptr : nullptr; }
mxLogical *mxGetLogicals(const mxArray *a) { return mxIsLogical(a) && !a->gpu ? (mxLogical *)a->data->ptr : nullptr; }

double mxGetScalar(const mxArray *a) {
    require_host(a, "mxGetScalar");
    if (a->kind != mxArray::NUMERIC || count(a->dims) == 0) return 0.0;
    const void *p = a->data->ptr;
    switch (a->cls) {
        case mxDOUBLE_CLASS: return *(const double *)p;
        case mxSINGLE_CLASS: return *(const float *)p;
        case mxLOGICAL_CLASS: return *(const mxLogical *)p ? 1.0 : 0.0;
        case mxINT8_CLASS: return *(const int8_t *)p;
        case mxUINT8_CLASS: return *(const uint8_t *)p;
        case mxINT16_CLASS: return *(const int16_t *)p;
        case mxUINT16_CLASS: return *(const uint16_t *)p;
        case mxINT32_CLASS: return *(const int32_t *)p;
        case mxUINT32_CLASS: return *(const uint32_t *)p;
        case mxINT64_CLASS: return (double)*(const int64_t *)p;
        case mxUINT64_CLASS: return (double)*(const uint64_t *)p;
        default: return 0.0;
    }
}

char *mxArrayToString(const mxArray *a) {
    if (!mxIsChar(a)) return nullptr;
    char *s = (char *)std::malloc(a->text.size() + 1);
    std::memcpy(s, a->text.c_str(), a->text.size() + 1);
    return s;
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
    char buf[2048];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw MexError(id ? id : "", buf);
}

void mexErrMsgTxt(const char *msg) { throw MexError("", msg ? msg : ""); }

void mexWarnMsgIdAndTxt(const char *id, const char *fmt, ...) {
    char buf[2048];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    std::fprintf(stderr, "Warning (%s): %s\n", id ? id : "", buf);
}

int mexAtExit(void (*fn)(void)) {
    for (auto h : exit_hooks())
        if (h == fn) return 0;
    exit_hooks().push_back(fn);
    return 0;
}

void mexLock(void) {}
void mexUnlock(void) {}

// -- gpuArray ---------------------------------------------------------------

int mxInitGPU(void) { return cudaFree(nullptr) == cudaSuccess ? MX_GPU_SUCCESS : MX_GPU_FAILURE; }

bool mxIsGPUArray(const mxArray *a) { return a && a->gpu; }

const mxGPUArray *mxGPUCreateFromMxArray(const mxArray *a) {
    if (!a || a->kind != mxArray::NUMERIC) throw MexError("parallel:gpu:array:InvalidInput", "not a numeric array");
    auto *g = new mxGPUArray;
    g->cls = a->cls;
    g->cplx = a->cplx;
    g->dims = a->dims;
    if (a->gpu) {
        g->data = a->data;                           // shares the gpuArray's memory, as MATLAB does
    } else {
        g->data = device_buffer(a->bytes(), false);  // a host array is copied to the device
        if (a->bytes()) cudaMemcpy(g->data->ptr, a->data->ptr, a->bytes(), cudaMemcpyHostToDevice);
    }
    return g;
}

mxGPUArray *mxGPUCopyFromMxArray(const mxArray *a) {
    const mxGPUArray *src = mxGPUCreateFromMxArray(a);
    auto *g = new mxGPUArray(*src);
    const size_t bytes = count(src->dims) * element_bytes(src->cls) * (src->cplx == mxCOMPLEX ? 2 : 1);
    g->data = device_buffer(bytes, false);
    if (bytes) cudaMemcpy(g->data->ptr, src->data->ptr, bytes, cudaMemcpyDeviceToDevice);
    delete src;
    return g;
}

mxGPUArray *mxGPUCreateGPUArray(mwSize ndim, const mwSize *dims, mxClassID cls, mxComplexity cplx,
                                mxGPUInitialize init) {
    auto *g = new mxGPUArray;
    g->cls = cls;
    g->cplx = cplx;
    g->dims = normalise(ndim, dims);
    const size_t bytes = count(g->dims) * element_bytes(cls) * (cplx == mxCOMPLEX ? 2 : 1);
    g->data = device_buffer(bytes, init == MX_GPU_INITIALIZE_VALUES);
    return g;
}

mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *g) {
    auto *a = new mxArray;
    a->gpu = true;
    a->cls = g->cls;
    a->cplx = g->cplx;
    a->dims = g->dims;
    a->data = g->data;
    return a;
}

void mxGPUDestroyGPUArray(const mxGPUArray *g) { delete g; }
mxClassID mxGPUGetClassID(const mxGPUArray *g) { return g->cls; }
mxComplexity mxGPUGetComplexity(const mxGPUArray *g) { return g->cplx; }
void *mxGPUGetData(mxGPUArray *g) { return g->data->ptr; }
const void *mxGPUGetDataReadOnly(const mxGPUArray *g) { return g->data->ptr; }

const mwSize *mxGPUGetDimensions(const mxGPUArray *g) {
    auto *d = (mwSize *)std::malloc(g->dims.size() * sizeof(mwSize));
    std::memcpy(d, g->dims.data(), g->dims.size() * sizeof(mwSize));
    return d;
}

mwSize mxGPUGetNumberOfDimensions(const mxGPUArray *g) { return g->dims.size(); }
mwSize mxGPUGetNumberOfElements(const mxGPUArray *g) { return count(g->dims); }

// -- driver entry points (the host side of the stand-in) ---------------------

// A gpuArray over existing device memory that the caller keeps alive.
mxArray *mexshim_gpu_wrap(void *ptr, int ndim, const size_t *dims, int cls, int cplx) {
    auto *a = new mxArray;
    a->gpu = true;
    a->cls = (mxClassID)cls;
    a->cplx = (mxComplexity)cplx;
    a->dims = normalise((size_t)ndim, dims);
    a->data = std::make_shared<Buffer>();
    a->data->ptr = ptr;
    a->data->device = true;
    a->data->owned = false;
    a->data->bytes = a->bytes();
    return a;
}

// A host array holding a copy of ``data`` (column-major, interleaved complex).
mxArray *mexshim_host_array(int ndim, const size_t *dims, int cls, int cplx, const void *data) {
    mxArray *a = numeric(normalise((size_t)ndim, dims), (mxClassID)cls, (mxComplexity)cplx);
    if (data && a->bytes()) std::memcpy(a->data->ptr, data, a->bytes());
    return a;
}

mxArray *mexshim_string(const char *s) { return mxCreateString(s); }

// A 1 x 1 struct that takes ownership of ``values``.
mxArray *mexshim_struct(int nfields, const char **names, mxArray **values) {
    mxArray *s = mxCreateStructMatrix(1, 1, nfields, names);
    for (int i = 0; i < nfields; ++i) s->values[i] = values[i];
    return s;
}

typedef void (*mex_function_t)(int, mxArray **, int, const mxArray **);

// Calls a MEX function.  Returns 0 on success, 1 when it raised an error
// through mexErrMsgIdAndTxt (identifier and message copied out), 2 on any
// other C++ exception.  Outputs the function created are left in plhs.
int mexshim_call(void *fn, int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs, char *id, char *msg,
                 int cap) {
    auto copy = [&](const std::string &i, const std::string &m) {
        if (cap > 0) {
            std::snprintf(id, (size_t)cap, "%s", i.c_str());
            std::snprintf(msg, (size_t)cap, "%s", m.c_str());
        }
    };
    for (int i = 0; i < nlhs; ++i) plhs[i] = nullptr;
    try {
        ((mex_function_t)fn)(nlhs, plhs, nrhs, prhs);
        return 0;
    } catch (const MexError &e) {
        copy(e.id, e.what());
        return 1;
    } catch (const std::exception &e) {
        copy("mexshim:exception", e.what());
        return 2;
    }
}

int mexshim_info(const mxArray *a, int *is_gpu, int *cls, int *cplx, int *ndim, size_t *dims, int cap) {
    if (!a) return -1;
    *is_gpu = a->gpu ? 1 : 0;
    *cls = (int)a->cls;
    *cplx = (int)a->cplx;
    *ndim = (int)a->dims.size();
    for (int i = 0; i < cap && i < (int)a->dims.size(); ++i) dims[i] = a->dims[i];
    return a->kind;
}

void *mexshim_data(const mxArray *a) { return a && a->data ? a->data->ptr : nullptr; }
mxArray *mexshim_field(const mxArray *s, const char *name) { return mxGetField(s, 0, name); }
void mexshim_destroy(mxArray *a) { delete a; }

// Device bytes currently owned by gpuArrays of the stand-in (leak checks).
long long mexshim_live_device_bytes(void) { return Buffer::live_device_bytes(0); }

// Runs the functions registered with mexAtExit, as `clear mex` would.
int mexshim_clear(void) {
    auto hooks = exit_hooks();
    exit_hooks().clear();
    for (auto it = hooks.rbegin(); it != hooks.rend(); ++it) (*it)();
    return (int)hooks.size();
}

}  // extern "C"
