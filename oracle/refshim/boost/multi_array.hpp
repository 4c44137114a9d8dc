// boost/multi_array.hpp stand-in (TEST INFRASTRUCTURE, see qshim.h): the
// three-dimensional array of doubles the reference's World keeps its
// distance, interaction and coupling tables in -- extents[a][b][c], resize,
// and [i][j][k] indexing in row-major order (Boost's default).
#pragma once

#include <cstddef>
#include <vector>

namespace boost {

struct extent3 { size_t a, b, c; };
struct extent2 {
    size_t a, b;
    extent3 operator[](size_t c) const { return extent3{a, b, c}; }
};
struct extent1 {
    size_t a;
    extent2 operator[](size_t b) const { return extent2{a, b}; }
};
struct extent_gen {
    extent1 operator[](size_t a) const { return extent1{a}; }
};
static const extent_gen extents = extent_gen();

template <class T, size_t N>
class multi_array;

template <class T>
class multi_array<T, 3> {
public:
    multi_array() {}
    explicit multi_array(const extent3& e) { resize(e); }
    // Boost keeps the elements whose indices survive a resize; the compiled
    // files resize empty arrays once, so a fresh zero-filled array is the same
    multi_array& resize(const extent3& e) {
        m_n1 = e.b;
        m_n2 = e.c;
        m_n0 = e.a;
        m_d.assign(e.a * e.b * e.c, T());
        return *this;
    }
    struct Row2 {
        T* p;
        T& operator[](size_t k) const { return p[k]; }
    };
    struct Row1 {
        T* p;
        size_t n2;
        Row2 operator[](size_t j) const { return Row2{p + j * n2}; }
    };
    Row1 operator[](size_t i) { return Row1{m_d.data() + i * m_n1 * m_n2, m_n2}; }
    size_t num_elements() const { return m_d.size(); }
    T* data() { return m_d.data(); }

private:
    std::vector<T> m_d;
    size_t m_n0 = 0, m_n1 = 0, m_n2 = 0;
};

}  // namespace boost
