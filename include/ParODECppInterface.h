/*
 * ParODECppInterface.h -- the C++ API of ParODE.
 *
 * Drop-in for the reference's Include/ParODECppInterface.h:22-57 (bodies
 * Sources/ParODE.cpp:176-242): the same function names and parameter lists on
 * `matrixf` / `vectorf`.  When Boost.uBLAS is on the include path the typedefs
 * are the reference's (boost::numeric::ublas::matrix<fType> / vector<fType>);
 * otherwise a source-compatible shim providing what callers use (size1, size2,
 * operator(), operator[], resize, element constructor) takes their place.
 *
 * The functions are inline wrappers over the C ABI of ParODECInterface.h, so
 * the library's binary interface does not depend on which matrix type the
 * caller compiles with.
 */
#ifndef PARODECPPINTERFACE_H_
#define PARODECPPINTERFACE_H_

#include <FTypeDef.h>
#include <ParODEEnums.h>
#include <ParODECInterface.h>
#include <parode_ext.h>

#include <cstddef>
#include <string>
#include <vector>

#if defined(__has_include)
#if __has_include(<boost/numeric/ublas/matrix.hpp>) && !defined(PARODE_NO_BOOST)
#define PARODE_HAVE_BOOST_UBLAS 1
#endif
#endif

#ifdef PARODE_HAVE_BOOST_UBLAS
#include <boost/numeric/ublas/matrix.hpp>
#include <boost/numeric/ublas/vector.hpp>
typedef boost::numeric::ublas::matrix<fType> matrixf;
typedef boost::numeric::ublas::vector<fType> vectorf;
#else
namespace parode_ublas_shim {
/* Row-major dense matrix with the uBLAS members ParODE callers use. */
template <class T>
class matrix {
public:
    matrix() : r_(0), c_(0) {}
    matrix(std::size_t r, std::size_t c) : r_(r), c_(c), d_(r * c) {}
    matrix(std::size_t r, std::size_t c, const T& v) : r_(r), c_(c), d_(r * c, v) {}
    std::size_t size1() const { return r_; }
    std::size_t size2() const { return c_; }
    void resize(std::size_t r, std::size_t c, bool preserve = true)
    {
        std::vector<T> nd(r * c, T());
        if (preserve)
            for (std::size_t i = 0; i < r && i < r_; ++i)
                for (std::size_t j = 0; j < c && j < c_; ++j) nd[i * c + j] = d_[i * c_ + j];
        d_.swap(nd);
        r_ = r;
        c_ = c;
    }
    T& operator()(std::size_t i, std::size_t j) { return d_[i * c_ + j]; }
    const T& operator()(std::size_t i, std::size_t j) const { return d_[i * c_ + j]; }
    T* data() { return d_.data(); }
    const T* data() const { return d_.data(); }

private:
    std::size_t r_, c_;
    std::vector<T> d_;
};

template <class T>
class vector {
public:
    vector() {}
    explicit vector(std::size_t n) : d_(n) {}
    vector(std::size_t n, const T& v) : d_(n, v) {}
    std::size_t size() const { return d_.size(); }
    void resize(std::size_t n, bool preserve = true)
    {
        if (!preserve) d_.assign(n, T());
        else d_.resize(n);
    }
    T& operator()(std::size_t i) { return d_[i]; }
    const T& operator()(std::size_t i) const { return d_[i]; }
    T& operator[](std::size_t i) { return d_[i]; }
    const T& operator[](std::size_t i) const { return d_[i]; }
    T* data() { return d_.data(); }
    const T* data() const { return d_.data(); }

private:
    std::vector<T> d_;
};
}  // namespace parode_ublas_shim
typedef parode_ublas_shim::matrix<fType> matrixf;
typedef parode_ublas_shim::vector<fType> vectorf;
#endif

/* Reference ParODECppInterface.h:167-168. */
inline ErrorCode InitializeAllGPUs(std::string& strKernelFolder, std::string& strIncludeFolder)
{
    int e = 0;
    std::vector<char> k(strKernelFolder.begin(), strKernelFolder.end()), i(strIncludeFolder.begin(),
                                                                              strIncludeFolder.end());
    k.push_back(0);
    i.push_back(0);
    ::InitializeAllGPUs(k.data(), i.data(), &e);
    return (ErrorCode)e;
}

/* Reference ParODECppInterface.h:170. */
inline ErrorCode GetAvailableGPUs(std::vector<unsigned int>& GPUIds)
{
    int n = 0, e = 0;
    int ids[64];
    ::GetAvailableGPUs(&n, ids, &e);
    GPUIds.clear();
    for (int q = 0; q < n && q < 64; ++q) GPUIds.push_back((unsigned int)ids[q]);
    return (ErrorCode)e;
}

/* Reference ParODECppInterface.h:172. */
inline ErrorCode GetDeviceName(unsigned int DeviceId, std::string& strDeviceName)
{
    int e = 0, id = (int)DeviceId;
    char buf[256];
    buf[0] = 0;
    ::GetDeviceName(&id, buf, &e);
    strDeviceName = buf;
    return (ErrorCode)e;
}

/* Reference ParODECppInterface.h:174-176. */
inline ErrorCode InitializeSelectedGPUs(const std::vector<unsigned int>& GPUIds, std::string& strKernelFolder,
                                        std::string& strIncludeFolder)
{
    int e = 0, n = (int)GPUIds.size();
    std::vector<int> ids(GPUIds.begin(), GPUIds.end());
    std::vector<char> k(strKernelFolder.begin(), strKernelFolder.end()), i(strIncludeFolder.begin(),
                                                                              strIncludeFolder.end());
    k.push_back(0);
    i.push_back(0);
    ::InitializeSelectedGPUs(&n, ids.data(), k.data(), i.data(), &e);
    return (ErrorCode)e;
}

/* Reference ParODECppInterface.h:179. */
inline void CloseGPU() { ::CloseGPUC(); }

/* Reference ParODECppInterface.h:182-183. */
inline ErrorCode StartTimer()
{
    int e = 0;
    ::StartTimer(&e);
    return (ErrorCode)e;
}
inline ErrorCode StopTimer(float& fTime)
{
    int e = 0;
    ::StopTimer(&fTime, &e);
    return (ErrorCode)e;
}

/* Reference ParODECppInterface.h:186. */
inline void GetErrorDescription(ErrorCode ErrNo, std::string& strErrDescription)
{
    int e = (int)ErrNo;
    char buf[256];
    ::GetErrorDescription(&e, buf);
    strErrDescription = buf;
}

/* Reference ParODECppInterface.h:190-199: xVect is resized to
 * (outputs x steps), tVect to (steps). */
inline ErrorCode SimulateODE(const matrixf& A, const matrixf& B, const matrixf& C, const matrixf& D, int uIndex,
                             double tStart, double tEnd, double tStep, const vectorf& x0, SolverType solver,
                             vectorf& tVect, matrixf& xVect)
{
    int n = (int)A.size1();
    int zB = B.size1() == 0 ? 1 : 0, zC = C.size1() == 0 ? 1 : 0, zD = D.size1() == 0 ? 1 : 0;
    int m = zB ? (zD ? 0 : (int)D.size2()) : (int)B.size2();
    int p = zC ? (zD ? n : (int)D.size1()) : (int)C.size1();
    std::vector<fType> a((std::size_t)n * n), b((std::size_t)n * (m > 0 ? m : 1)),
        c((std::size_t)(p > 0 ? p : 1) * n), d((std::size_t)(p > 0 ? p : 1) * (m > 0 ? m : 1)), x((std::size_t)n);
    for (int r = 0; r < n; ++r)
        for (int q = 0; q < n; ++q) a[(std::size_t)r * n + q] = A(r, q);
    if (!zB)
        for (int r = 0; r < n; ++r)
            for (int q = 0; q < m; ++q) b[(std::size_t)r * m + q] = B(r, q);
    if (!zC)
        for (int r = 0; r < p; ++r)
            for (int q = 0; q < n; ++q) c[(std::size_t)r * n + q] = C(r, q);
    if (!zD)
        for (int r = 0; r < p; ++r)
            for (int q = 0; q < m; ++q) d[(std::size_t)r * m + q] = D(r, q);
    for (int r = 0; r < n && r < (int)x0.size(); ++r) x[(std::size_t)r] = x0(r);
    int solv = (int)solver;
    long long T = ParODE_NumOutputs(solv, tStart, tEnd, tStep);
    if (T <= 0) return ParODE_InvalidSystem;
    std::vector<fType> tv((std::size_t)T), yv((std::size_t)T * (p > 0 ? p : 1));
    int e = 0, nSteps = 0, nIn = m, nSt = n, nOut = p, ui = uIndex;
    ::SimulateODE(a.data(), b.data(), c.data(), d.data(), &nIn, &nSt, &nOut, &zB, &zC, &zD, &ui, &tStart, &tEnd,
                  &tStep, x.data(), &solv, tv.data(), yv.data(), &nSteps, &e);
    if (e != 0) return (ErrorCode)e;
    tVect.resize((std::size_t)nSteps);
    xVect.resize((std::size_t)p, (std::size_t)nSteps);
    for (int k = 0; k < nSteps; ++k) {
        tVect[(std::size_t)k] = tv[(std::size_t)k];
        for (int r = 0; r < p; ++r) xVect(r, k) = yv[(std::size_t)k * p + r];
    }
    return ParODE_OK;
}

/* Reference ParODECppInterface.h:202. */
inline int RegisterInput(const std::string& uFunc)
{
    std::vector<char> s(uFunc.begin(), uFunc.end());
    s.push_back(0);
    int idx = -1, e = 0;
    ::RegisterInput(s.data(), &idx, &e);
    return e != 0 ? e : idx;
}

#endif /* PARODECPPINTERFACE_H_ */
