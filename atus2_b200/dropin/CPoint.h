// CPoint.h (drop-in) -- position / momentum vectors of dim doubles with the
// interface of ATUS-2's CPoint<dim> (include/CPoint.h:36-183): zero-filled
// default, initializer-list construction, element access, component-wise
// += -= and scalar *= /=, + and - of two points, scale (component-wise
// product), the dot product as operator*, comparison with a scalar and Dump /
// operator<< as "a,b,c".  Differences: operator*(double) returns the scaled
// point (the reference assigns the last component's product to every
// component), and the index check rejects index == dim as well.
#ifndef ATUS_DROPIN_CPOINT_H
#define ATUS_DROPIN_CPOINT_H

#include <initializer_list>
#include <iostream>
#include <string>
#include <vector>

template <int dim>
class CPoint {
 public:
  CPoint() {
    for (int i = 0; i < dim; i++) m_data[i] = 0;
  }
  CPoint(std::initializer_list<double> list) {
    if ((int)list.size() != dim) throw std::string("Error: initializer_list size mismatch\n");
    int i = 0;
    for (double v : list) m_data[i++] = v;
  }
  CPoint &operator=(const double s) {
    for (int i = 0; i < dim; i++) m_data[i] = s;
    return *this;
  }
  CPoint &operator=(const std::vector<double> &vec) {
    for (int i = 0; i < dim; i++) m_data[i] = vec[i];
    return *this;
  }
  double &operator[](int index) {
    if (index < 0 || index >= dim) throw std::string("Error: Index out of bound\n");
    return m_data[index];
  }
  const double &operator[](int index) const {
    if (index < 0 || index >= dim) throw std::string("Error: Index out of bound\n");
    return m_data[index];
  }
  CPoint &operator+=(const CPoint &r) {
    for (int i = 0; i < dim; i++) m_data[i] += r.m_data[i];
    return *this;
  }
  CPoint &operator-=(const CPoint &r) {
    for (int i = 0; i < dim; i++) m_data[i] -= r.m_data[i];
    return *this;
  }
  CPoint &operator*=(const double s) {
    for (int i = 0; i < dim; i++) m_data[i] *= s;
    return *this;
  }
  CPoint &operator/=(const double s) {
    for (int i = 0; i < dim; i++) m_data[i] /= s;
    return *this;
  }
  CPoint operator+(const CPoint &r) const {
    CPoint out(*this);
    out += r;
    return out;
  }
  CPoint operator-(const CPoint &r) const {
    CPoint out(*this);
    out -= r;
    return out;
  }
  CPoint scale(const CPoint &b) const {
    CPoint out;
    for (int i = 0; i < dim; i++) out.m_data[i] = m_data[i] * b.m_data[i];
    return out;
  }
  double operator*(const CPoint &r) const {
    double s = 0;
    for (int i = 0; i < dim; i++) s += m_data[i] * r.m_data[i];
    return s;
  }
  CPoint operator*(double s) const {
    CPoint out(*this);
    out *= s;
    return out;
  }
  bool operator==(const double s) const {
    for (int i = 0; i < dim; i++)
      if (m_data[i] != s) return false;
    return true;
  }
  void Dump(std::ostream &os) const {
    for (int i = 0; i < dim; i++) os << m_data[i] << ((i == dim - 1) ? "" : ",");
  }
  double *data() { return m_data; }
  const double *data() const { return m_data; }

 protected:
  double m_data[dim];
};

template <int dim>
std::ostream &operator<<(std::ostream &os, const CPoint<dim> &p) {
  p.Dump(os);
  return os;
}

#endif
