// Minimal stand-in for the small part of the OpenCV C++ API that the
// reference's legacy dense code (opensfm/src/lib/dense/src/depthmap.cc and
// opensfm/src/lib/dense/depthmap.h) uses, so that file compiles unmodified
// as a CPU oracle.  TEST INFRASTRUCTURE ONLY: nothing in the product links it.
//
// Written for this project from the documented OpenCV 4.x semantics (the
// version the reference pins is libopencv 4.13.0).  Arithmetic follows those
// semantics where results depend on it:
//   * Matx * Matx accumulates in the element type, starting from 0, k = 0..l-1.
//   * scalar * Matx / Matx * scalar / Vec * scalar compute a[i] * alpha in the
//     wider of the two types and round back to the element type.
//   * Vec / float multiplies by the float reciprocal 1.f / alpha.
//   * Matx<T,3,3>::inv() uses the cofactor form scaled by 1 / det.
//   * normalize(Vec) divides by the double L2 norm (multiply by 1./norm).
//   * medianBlur(CV_32F, 5) is the exact 5x5 median with replicated borders.
// The shim's inv() and medianBlur() are checked against Python cv2 4.13 by
// tests/test_oracle.py.
#pragma once

#include <math.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

#define CV_8U 0
#define CV_32S 4
#define CV_32F 5
#define CV_8UC3 16
#define CV_32FC3 21

namespace cv {

template <typename T>
struct Scalar_ {
  T val[4];
  Scalar_(T v0 = 0, T v1 = 0, T v2 = 0, T v3 = 0) {
    val[0] = v0;
    val[1] = v1;
    val[2] = v2;
    val[3] = v3;
  }
};
typedef Scalar_<double> Scalar;

template <typename T, int m, int n>
struct Matx {
  enum { rows = m, cols = n, channels = m * n };
  T val[m * n];

  Matx() {
    for (int i = 0; i < m * n; ++i) val[i] = T(0);
  }
  explicit Matx(const T* vals) {
    for (int i = 0; i < m * n; ++i) val[i] = vals[i];
  }
  Matx(T v0, T v1, T v2) {
    static_assert(m * n == 3, "3-element constructor");
    val[0] = v0;
    val[1] = v1;
    val[2] = v2;
  }
  template <typename T2>
  operator Matx<T2, m, n>() const {
    Matx<T2, m, n> r;
    for (int i = 0; i < m * n; ++i) r.val[i] = static_cast<T2>(val[i]);
    return r;
  }
  T& operator()(int i, int j) { return val[i * n + j]; }
  const T& operator()(int i, int j) const { return val[i * n + j]; }
  T& operator()(int i) { return val[i]; }
  const T& operator()(int i) const { return val[i]; }

  Matx<T, n, m> t() const {
    Matx<T, n, m> r;
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < n; ++j) r.val[j * m + i] = val[i * n + j];
    return r;
  }
  T dot(const Matx<T, m, n>& o) const {
    T s = 0;
    for (int i = 0; i < m * n; ++i) s += val[i] * o.val[i];
    return s;
  }
  Matx<T, m, n> inv() const;
};

template <typename T, int m, int n>
Matx<T, m, n> Matx<T, m, n>::inv() const {
  static_assert(m == 3 && n == 3, "shim only inverts 3x3");
  const Matx& a = *this;
  T d = a(0, 0) * (a(1, 1) * a(2, 2) - a(2, 1) * a(1, 2)) -
        a(0, 1) * (a(1, 0) * a(2, 2) - a(2, 0) * a(1, 2)) +
        a(0, 2) * (a(1, 0) * a(2, 1) - a(2, 0) * a(1, 1));
  Matx r;
  if (d == 0) return r;
  d = 1 / d;
  r(0, 0) = (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) * d;
  r(0, 1) = (a(0, 2) * a(2, 1) - a(0, 1) * a(2, 2)) * d;
  r(0, 2) = (a(0, 1) * a(1, 2) - a(0, 2) * a(1, 1)) * d;
  r(1, 0) = (a(1, 2) * a(2, 0) - a(1, 0) * a(2, 2)) * d;
  r(1, 1) = (a(0, 0) * a(2, 2) - a(0, 2) * a(2, 0)) * d;
  r(1, 2) = (a(0, 2) * a(1, 0) - a(0, 0) * a(1, 2)) * d;
  r(2, 0) = (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0)) * d;
  r(2, 1) = (a(0, 1) * a(2, 0) - a(0, 0) * a(2, 1)) * d;
  r(2, 2) = (a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0)) * d;
  return r;
}

template <typename T, int cn>
struct Vec : public Matx<T, cn, 1> {
  typedef Matx<T, cn, 1> Base;
  Vec() : Base() {}
  explicit Vec(const T* vals) : Base(vals) {}
  Vec(T v0, T v1, T v2) : Base(v0, v1, v2) {}
  Vec(const Base& b) : Base(b) {}
  template <typename T2>
  operator Vec<T2, cn>() const {
    Vec<T2, cn> r;
    for (int i = 0; i < cn; ++i) r.val[i] = static_cast<T2>(this->val[i]);
    return r;
  }
  T& operator[](int i) { return this->val[i]; }
  const T& operator[](int i) const { return this->val[i]; }
};

typedef Matx<float, 3, 3> Matx33f;
typedef Matx<double, 3, 3> Matx33d;
typedef Vec<float, 3> Vec3f;
typedef Vec<double, 3> Vec3d;
typedef Vec<unsigned char, 3> Vec3b;

// Matrix product, accumulating in T from zero.
template <typename T, int m, int l, int n>
Matx<T, m, n> operator*(const Matx<T, m, l>& a, const Matx<T, l, n>& b) {
  Matx<T, m, n> r;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) {
      T s = 0;
      for (int k = 0; k < l; ++k) s += a(i, k) * b(k, j);
      r(i, j) = s;
    }
  return r;
}
template <typename T, int m, int n>
Vec<T, m> operator*(const Matx<T, m, n>& a, const Vec<T, n>& b) {
  const Matx<T, n, 1>& bb = b;
  return Vec<T, m>(a * bb);
}
template <typename T, int m, int n>
Matx<T, m, n> operator+(const Matx<T, m, n>& a, const Matx<T, m, n>& b) {
  Matx<T, m, n> r;
  for (int i = 0; i < m * n; ++i) r.val[i] = static_cast<T>(a.val[i] + b.val[i]);
  return r;
}
template <typename T, int cn>
Vec<T, cn> operator+(const Vec<T, cn>& a, const Vec<T, cn>& b) {
  Vec<T, cn> r;
  for (int i = 0; i < cn; ++i) r.val[i] = static_cast<T>(a.val[i] + b.val[i]);
  return r;
}
template <typename T, int cn>
Vec<T, cn> operator-(const Vec<T, cn>& a, const Vec<T, cn>& b) {
  Vec<T, cn> r;
  for (int i = 0; i < cn; ++i) r.val[i] = static_cast<T>(a.val[i] - b.val[i]);
  return r;
}
// Scaling: the product is formed in the wider type, then rounded to T.
template <typename T, int m, int n>
Matx<T, m, n> operator*(float alpha, const Matx<T, m, n>& a) {
  Matx<T, m, n> r;
  for (int i = 0; i < m * n; ++i) r.val[i] = static_cast<T>(a.val[i] * alpha);
  return r;
}
template <typename T, int m, int n>
Matx<T, m, n> operator*(double alpha, const Matx<T, m, n>& a) {
  Matx<T, m, n> r;
  for (int i = 0; i < m * n; ++i) r.val[i] = static_cast<T>(a.val[i] * alpha);
  return r;
}
template <typename T, int cn>
Vec<T, cn> operator*(const Vec<T, cn>& a, double alpha) {
  Vec<T, cn> r;
  for (int i = 0; i < cn; ++i) r.val[i] = static_cast<T>(a.val[i] * alpha);
  return r;
}
template <typename T, int cn>
Vec<T, cn> operator*(const Vec<T, cn>& a, float alpha) {
  Vec<T, cn> r;
  for (int i = 0; i < cn; ++i) r.val[i] = static_cast<T>(a.val[i] * alpha);
  return r;
}
template <typename T, int cn>
Vec<T, cn> operator/(const Vec<T, cn>& a, float alpha) {
  const float inv = 1.f / alpha;
  Vec<T, cn> r;
  for (int i = 0; i < cn; ++i) r.val[i] = static_cast<T>(a.val[i] * inv);
  return r;
}

template <typename T, int cn>
double norm(const Vec<T, cn>& v) {
  double s = 0;
  for (int i = 0; i < cn; ++i) {
    double x = v.val[i];
    s += x * x;
  }
  return std::sqrt(s);
}
template <typename T, int cn>
Vec<T, cn> normalize(const Vec<T, cn>& v) {
  double nv = norm(v);
  return v * (nv ? 1. / nv : 0.);
}

class Mat {
 public:
  int rows = 0, cols = 0;

  Mat() = default;
  Mat(int r, int c, int type, void* data) : rows(r), cols(c), type_(type) {
    elem_ = elem_size(type);
    ext_ = static_cast<unsigned char*>(data);
  }
  Mat(int r, int c, int type, const Scalar& s) : rows(r), cols(c), type_(type) {
    elem_ = elem_size(type);
    own_ = std::make_shared<std::vector<unsigned char>>(size_t(r) * c * elem_);
    const int ch = channels(type);
    for (int i = 0; i < r * c; ++i)
      for (int k = 0; k < ch; ++k) set_channel(i, k, s.val[k]);
  }
  Mat clone() const {
    Mat m;
    m.rows = rows;
    m.cols = cols;
    m.type_ = type_;
    m.elem_ = elem_;
    m.own_ = std::make_shared<std::vector<unsigned char>>(bytes());
    if (bytes()) std::memcpy(m.own_->data(), data(), bytes());
    return m;
  }
  int type() const { return type_; }
  unsigned char* data() const { return own_ ? own_->data() : ext_; }
  size_t bytes() const { return size_t(rows) * cols * elem_; }
  template <typename T>
  T& at(int i, int j) {
    return reinterpret_cast<T*>(data())[size_t(i) * cols + j];
  }
  template <typename T>
  const T& at(int i, int j) const {
    return reinterpret_cast<const T*>(data())[size_t(i) * cols + j];
  }

 private:
  static size_t elem_size(int type) {
    switch (type) {
      case CV_8U: return 1;
      case CV_32S: return 4;
      case CV_32F: return 4;
      case CV_8UC3: return 3;
      case CV_32FC3: return 12;
    }
    throw std::runtime_error("opencv shim: unsupported Mat type");
  }
  static int channels(int type) { return (type == CV_8UC3 || type == CV_32FC3) ? 3 : 1; }
  void set_channel(int idx, int k, double v) {
    unsigned char* p = data() + size_t(idx) * elem_;
    switch (type_) {
      case CV_8U:
      case CV_8UC3: p[k] = static_cast<unsigned char>(v); break;
      case CV_32S: reinterpret_cast<int32_t*>(p)[k] = static_cast<int32_t>(v); break;
      case CV_32F:
      case CV_32FC3: reinterpret_cast<float*>(p)[k] = static_cast<float>(v); break;
    }
  }
  int type_ = CV_8U;
  size_t elem_ = 1;
  unsigned char* ext_ = nullptr;
  std::shared_ptr<std::vector<unsigned char>> own_;
};

// Exact median over a ksize x ksize window with replicated borders; the shim
// supports the single case the reference uses (CV_32F, ksize 5).
inline void medianBlur(const Mat& src, Mat& dst, int ksize) {
  if (src.type() != CV_32F || ksize != 5)
    throw std::runtime_error("opencv shim: medianBlur supports CV_32F, ksize 5");
  Mat out(src.rows, src.cols, CV_32F, Scalar(0));
  const int r = ksize / 2;
  std::vector<float> win(ksize * ksize);
  for (int i = 0; i < src.rows; ++i)
    for (int j = 0; j < src.cols; ++j) {
      int c = 0;
      for (int di = -r; di <= r; ++di)
        for (int dj = -r; dj <= r; ++dj) {
          int ii = std::min(std::max(i + di, 0), src.rows - 1);
          int jj = std::min(std::max(j + dj, 0), src.cols - 1);
          win[c++] = src.at<float>(ii, jj);
        }
      std::nth_element(win.begin(), win.begin() + c / 2, win.begin() + c);
      out.at<float>(i, j) = win[c / 2];
    }
  dst = out;
}

}  // namespace cv
