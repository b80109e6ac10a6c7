/* Stand-in for the TNT / JAMA headers the reference's surface_field.h
 * includes (surface_field.h:10-11; TNT and JAMA are not part of the
 * reference tree).  Test infrastructure only: it lets the reference's own
 * surface_field.cpp compile into the oracle build.  It provides the pieces
 * surface_field::surface_aniso uses (surface_field.cpp:91-92, 126-135):
 * TNT::Array1D / Array2D with operator[], and JAMA::SVD<T> with
 * getSingularValues / getU / getV, singular values in descending order.
 *
 * The decomposition is this repository's own: the matrices it is given are
 * symmetric covariance matrices, so it diagonalises them with cyclic Jacobi
 * rotations (the classical method: rotate the largest off-diagonal pairs to
 * zero until they vanish), takes |eigenvalue| as singular value, V = the
 * eigenvectors and U = V with the column negated where an eigenvalue is
 * negative.  A non-symmetric input is decomposed through A^T A the same way
 * (U = A V / s).  Results agree with any other SVD to rounding; surface_aniso
 * only uses U diag(1/s) V^T, which does not depend on the eigenvectors'
 * signs.  (marching_cubes.cpp also relies on a header for memcpy; the build
 * adds -include cstring.) */
#ifndef REFSHIM_JAMA_SVD_H_
#define REFSHIM_JAMA_SVD_H_
#include <cmath>
#include <vector>

namespace TNT {
template <class T>
class Array1D {
public:
    explicit Array1D(int n = 0) : d_(n) {}
    T& operator[](int i) { return d_[i]; }
    const T& operator[](int i) const { return d_[i]; }
    int dim() const { return (int)d_.size(); }
private:
    std::vector<T> d_;
};
template <class T>
class Array2D {
public:
    Array2D(int m = 0, int n = 0) : m_(m), n_(n), d_((size_t)m * n) {}
    T* operator[](int i) { return &d_[(size_t)i * n_]; }
    const T* operator[](int i) const { return &d_[(size_t)i * n_]; }
    int dim1() const { return m_; }
    int dim2() const { return n_; }
private:
    int m_, n_;
    std::vector<T> d_;
};
}  // namespace TNT

namespace JAMA {
template <class T>
class SVD {
public:
    explicit SVD(const TNT::Array2D<T>& A) {
        T a[3][3], s_in[3][3];
        bool sym = true;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                a[i][j] = A[i][j];
                if (A[i][j] != A[j][i]) sym = false;
            }
        if (sym) {
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) s_in[i][j] = a[i][j];
        } else {  // A^T A
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    T t = 0;
                    for (int k = 0; k < 3; ++k) t += a[k][i] * a[k][j];
                    s_in[i][j] = t;
                }
        }
        T ev[3], vec[3][3];
        jacobi(s_in, ev, vec);
        // order by |eigenvalue| (descending)
        int ord[3] = {0, 1, 2};
        for (int i = 0; i < 3; ++i)
            for (int j = i + 1; j < 3; ++j)
                if (std::fabs(ev[ord[j]]) > std::fabs(ev[ord[i]])) { int t = ord[i]; ord[i] = ord[j]; ord[j] = t; }
        for (int k = 0; k < 3; ++k) {
            const int o = ord[k];
            for (int i = 0; i < 3; ++i) v_[i][k] = vec[i][o];
            if (sym) {
                s_[k] = std::fabs(ev[o]);
                const T sg = ev[o] < 0 ? T(-1) : T(1);
                for (int i = 0; i < 3; ++i) u_[i][k] = sg * vec[i][o];
            } else {
                s_[k] = std::sqrt(std::fabs(ev[o]));
                for (int i = 0; i < 3; ++i) {
                    T t = 0;
                    for (int j = 0; j < 3; ++j) t += a[i][j] * vec[j][o];
                    u_[i][k] = s_[k] > 0 ? t / s_[k] : T(0);
                }
            }
        }
    }
    void getSingularValues(TNT::Array1D<T>& s) const { for (int i = 0; i < 3; ++i) s[i] = s_[i]; }
    void getU(TNT::Array2D<T>& U) const { for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) U[i][j] = u_[i][j]; }
    void getV(TNT::Array2D<T>& V) const { for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) V[i][j] = v_[i][j]; }

private:
    T s_[3], u_[3][3], v_[3][3];

    // cyclic Jacobi rotations on a symmetric 3x3 matrix m: eigenvalues ev,
    // eigenvectors as the columns of vec
    static void jacobi(T m[3][3], T ev[3], T vec[3][3]) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) vec[i][j] = i == j ? T(1) : T(0);
        for (int sweep = 0; sweep < 64; ++sweep) {
            const T off = std::fabs(m[0][1]) + std::fabs(m[0][2]) + std::fabs(m[1][2]);
            const T dia = std::fabs(m[0][0]) + std::fabs(m[1][1]) + std::fabs(m[2][2]);
            if (off == T(0) || off <= dia * T(1e-300)) break;
            for (int p = 0; p < 2; ++p)
                for (int q = p + 1; q < 3; ++q) {
                    if (m[p][q] == T(0)) continue;
                    const T theta = (m[q][q] - m[p][p]) / (T(2) * m[p][q]);
                    const T t = (theta >= 0 ? T(1) : T(-1)) / (std::fabs(theta) + std::sqrt(theta * theta + T(1)));
                    const T c = T(1) / std::sqrt(t * t + T(1)), s = t * c;
                    for (int k = 0; k < 3; ++k) {  // m <- m J
                        const T mkp = m[k][p], mkq = m[k][q];
                        m[k][p] = c * mkp - s * mkq;
                        m[k][q] = s * mkp + c * mkq;
                    }
                    for (int k = 0; k < 3; ++k) {  // m <- J^T m
                        const T mpk = m[p][k], mqk = m[q][k];
                        m[p][k] = c * mpk - s * mqk;
                        m[q][k] = s * mpk + c * mqk;
                    }
                    for (int k = 0; k < 3; ++k) {
                        const T vkp = vec[k][p], vkq = vec[k][q];
                        vec[k][p] = c * vkp - s * vkq;
                        vec[k][q] = s * vkp + c * vkq;
                    }
                }
        }
        for (int i = 0; i < 3; ++i) ev[i] = m[i][i];
    }
};
}  // namespace JAMA

// surface_field.cpp names std::vector unqualified, as the TNT / JAMA headers
// it was written against let it
using std::vector;
#endif
