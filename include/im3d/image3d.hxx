/*
 * image3d.hxx -- im3d::image3d<T>, the volume container of the header-only API, with
 * the public interface of the reference's class (header/image3d.hxx:50-765) for the
 * members on the segmentation path.
 *
 * Layout is the reference's (header/image3d_imp.hxx:142-153): (i, j, k) at
 * dimy*dimz*i + dimz*j + k, k contiguous, so data() can be handed to the C ABI as is.
 * Element-wise operators, scalar products and norms run on the host, on the host
 * buffer this class owns, with the reference's semantics (a size mismatch prints the
 * same WARNING and leaves the left operand unchanged). grad and div run on the B200
 * backend (im3d_grad_* / im3d_div_*). The processing utilities off the segmentation
 * path (crop, change_resolution, histogram_equalization, median_filter,
 * connected_component, ...) are not part of this backend.
 */
#ifndef IM3D_IMAGE3D_HXX
#define IM3D_IMAGE3D_HXX

#include <algorithm>
#include <cmath>
#include <iostream>
#include <vector>

#include "b200.hxx"
#include "names.hxx"

namespace im3d
{

template <typename T = double>
class image3d
{
protected:
    std::vector<T> rawimage;
    uint dimx = 0, dimy = 0, dimz = 0;
    double hx = 1., hy = 1., hz = 1.;

    template <typename S>
    friend class image3d;

public:
    image3d () {}
    image3d (uint const& x, uint const& y, uint const& z, double const& hx = 1.,
             double const& hy = 1., double const& hz = 1.)
        : rawimage ( (size_t) x * y * z, T (0) ), dimx (x), dimy (y), dimz (z), hx (hx), hy (hy),
          hz (hz)
    {
    }
    image3d (image3d const& tocopy) = default;
    virtual ~image3d () {}

    // ---- sizes and spacing (image3d.hxx:122-238)
    inline uint getdimx () const { return dimx; }
    inline uint getdimy () const { return dimy; }
    inline uint getdimz () const { return dimz; }
    inline double gethx () const { return hx; }
    inline double gethy () const { return hy; }
    inline double gethz () const { return hz; }
    inline void setdimx (uint const& x) { dimx = x; reset (T (0) ); }
    inline void setdimy (uint const& y) { dimy = y; reset (T (0) ); }
    inline void setdimz (uint const& z) { dimz = z; reset (T (0) ); }
    inline void setdim (uint const& x, uint const& y, uint const& z, T const& value = 0)
    {
        dimx = x;
        dimy = y;
        dimz = z;
        reset (value);
    }
    inline void sethx (double const& h) { hx = h; }
    inline void sethy (double const& h) { hy = h; }
    inline void sethz (double const& h) { hz = h; }
    inline void seth (double const& x, double const& y, double const& z)
    {
        hx = x;
        hy = y;
        hz = z;
    }

    // raw access for the C ABI (no counterpart in the reference, whose buffer is protected)
    inline T* data () { return rawimage.data(); }
    inline T const* data () const { return rawimage.data(); }
    inline size_t size () const { return rawimage.size(); }

    // ---- element access (image3d_imp.hxx:142-153)
    virtual inline T operator() (uint const& i, uint const& j, uint const& k) const
    {
        return rawimage[ (size_t) dimy * dimz * i + (size_t) dimz * j + k];
    }
    virtual inline T& operator() (uint const& i, uint const& j, uint const& k)
    {
        return rawimage[ (size_t) dimy * dimz * i + (size_t) dimz * j + k];
    }

    // ---- assignment and in-place arithmetic (image3d_imp.hxx:156-345)
    template <typename S>
    image3d<T>& operator= (S const& v)
    {
        std::fill (rawimage.begin(), rawimage.end(), static_cast<T> (v) );
        return *this;
    }
    template <typename S>
    image3d<T>& operator= (image3d<S> const& o)
    {
        dimx = o.dimx;
        dimy = o.dimy;
        dimz = o.dimz;
        hx = o.hx;
        hy = o.hy;
        hz = o.hz;
        rawimage.resize (o.rawimage.size() );
        for (size_t q = 0; q < rawimage.size(); ++q) rawimage[q] = static_cast<T> (o.rawimage[q]);
        return *this;
    }
    image3d<T>& operator= (image3d<T> const& o) = default;

    template <typename S> image3d<T>& operator+= (S const& v) { return scalar_op (v, 0); }
    template <typename S> image3d<T>& operator-= (S const& v) { return scalar_op (v, 1); }
    template <typename S> image3d<T>& operator*= (S const& v) { return scalar_op (v, 2); }
    template <typename S> image3d<T>& operator/= (S const& v) { return scalar_op (v, 3); }
    template <typename S> image3d<T>& operator+= (image3d<S> const& o) { return image_op (o, 0, "+="); }
    template <typename S> image3d<T>& operator-= (image3d<S> const& o) { return image_op (o, 1, "-="); }
    template <typename S> image3d<T>& operator*= (image3d<S> const& o) { return image_op (o, 2, "*="); }
    template <typename S> image3d<T>& operator/= (image3d<S> const& o) { return image_op (o, 3, "/="); }

    // ---- scalar products and norms (image3d_imp.hxx:385-428, 1388-1511)
    template <typename S, typename R>
    friend S const scalarprod (image3d<S> const& a, image3d<R> const& b);
    template <typename S, typename R>
    friend S const scalarprod_L2 (image3d<S> const& a, image3d<R> const& b);

    T const norm1 () const
    {
        T s = 0;
        for (T v : rawimage) s += std::abs (v);
        return s;
    }
    T const normL1 () const { return norm1() * hx * hy * hz; }
    T const norm2 () const { return std::sqrt (scalarprod (*this, *this) ); }
    T const normL2 () const { return std::sqrt (scalarprod_L2 (*this, *this) ); }
    // the reference compares the signed value and keeps its magnitude (:1428-1453)
    T const norminf () const
    {
        if (rawimage.empty() ) return T (0);
        T m = std::abs (rawimage[0]);
        for (T v : rawimage)
            if (m < v) m = std::abs (v);
        return m;
    }
    T const max () const
    {
        if (rawimage.empty() ) return T (0);
        T m = rawimage[0];
        for (T v : rawimage)
            if (m < v) m = v;
        return m;
    }
    T const min () const
    {
        if (rawimage.empty() ) return T (0);
        T m = rawimage[0];
        for (T v : rawimage)
            if (m > v) m = v;
        return m;
    }

    // affine map [min, max] -> [min', max'] (image3d_imp.hxx:1628-1636)
    void change_range_of_intensity (T const& mx, T const& mn = 0)
    {
        (*this) -= this->min();
        (*this) /= this->max() / (mx - mn);
        (*this) += mn;
    }

    // ---- differential operators on the B200 backend (image3d_imp.hxx:744-1384)
    template <typename S>
    void grad (std::vector<image3d<S> >& res) const
    {
        if (dimz <= 1)
        {
            std::clog << "WARNING::image3d::grad: 2-D images are not supported by the B200 "
                      << "backend" << std::endl;
            return;
        }
        std::vector<T> out (3 * rawimage.size() );
        if (b200::failed (b200::ops<T>::grad (b200::context(), rawimage.data(), out.data(), dimx,
                                              dimy, dimz, hx, hy, hz), "image3d::grad") )
            return;
        res.resize (3);
        for (int c = 0; c < 3; ++c)
        {
            res[c].setdim (dimx, dimy, dimz);
            res[c].seth (hx, hy, hz);
            for (size_t q = 0; q < rawimage.size(); ++q)
                res[c].rawimage[q] = static_cast<S> (out[c * rawimage.size() + q]);
        }
    }

    // black and white image (image3d_imp.hxx:1592-1623): 1 where the image is at or
    // above min + (max - min) * threshold, 0 elsewhere (the other way round if negative)
    template <typename S>
    void im_to_black_and_white (image3d<S>& res, double threshold = 0.5,
                                bool negative = false) const
    {
        if (threshold > 1 || threshold < 0)
        {
            std::cout << "WARNING::im_to_black_and_white: threshold must be between 0 and 1, ";
            std::cout << "otherwise default value 0.5 is applied" << std::endl;
            threshold = 0.5;
        }
        const T mx (this->max() ), mn (this->min() ), pivot (mn + (mx - mn) * threshold);
        res.setdim (dimx, dimy, dimz);
        res.seth (hx, hy, hz);
        for (size_t q = 0; q < rawimage.size(); ++q)
            res.rawimage[q] = static_cast<S> (rawimage[q] < pivot ? int (negative) : 1 - int (negative) );
    }

    // ---- connected components on the B200 backend (image3d_imp.hxx:1694-2120)
    // the component containing cell (i, j, k) of the black and white image
    template <typename S>
    void connected_component (image3d<S>& res, uint const& i, uint const& j, uint const& k,
                              double threshold = 0.5, bool full_connected = false,
                              bool binary_output = true) const
    {
        cc_backend (res, nullptr, (int) i, (int) j, (int) k, threshold, full_connected, binary_output);
    }

    // the cells connected to the non-zero cells of init that are white
    template <typename S>
    void connected_component (image3d<S>& res, image3d<S> const& init, double threshold = 0.5,
                              bool full_connected = false, bool binary_output = true) const
    {
        if (init.getdimx() != dimx || init.getdimy() != dimy || init.getdimz() != dimz)
        {
            std::cout << "WARNING: in image3d::connected_component: dimensions of init must be ";
            std::cout << "the same of the image" << std::endl;
            return;
        }
        std::vector<T> ini (rawimage.size() );
        for (size_t q = 0; q < ini.size(); ++q) ini[q] = static_cast<T> (init.rawimage[q] != S (0) );
        cc_backend (res, ini.data(), 0, 0, 0, threshold, full_connected, binary_output);
    }

    template <typename S, typename R>
    friend void vector_abs (image3d<S>& res, std::vector<image3d<R> > const& fun);
    template <typename S, typename R>
    friend void div (image3d<S>& res, std::vector<image3d<R> > const& fun);

private:
    template <typename S>
    void cc_backend (image3d<S>& res, T const* init, int i, int j, int k, double threshold,
                     bool full_connected, bool binary_output) const
    {
        std::vector<T> out (rawimage.size() );
        if (b200::failed (b200::ops<T>::cc (b200::context(), rawimage.data(), out.data(), dimx, dimy,
                                            dimz, init, i, j, k, threshold, full_connected ? 1 : 0,
                                            binary_output ? 1 : 0), "image3d::connected_component") )
            return;
        res.setdim (dimx, dimy, dimz);
        res.seth (hx, hy, hz);
        for (size_t q = 0; q < out.size(); ++q) res.rawimage[q] = static_cast<S> (out[q]);
    }

    void reset (T const& value)
    {
        rawimage.assign ( (size_t) dimx * dimy * dimz, value);
    }

    template <typename S>
    image3d<T>& scalar_op (S const& v, int op)
    {
        const T s = static_cast<T> (v);
        for (T& x : rawimage)
        {
            if (op == 0) x += s;
            else if (op == 1) x -= s;
            else if (op == 2) x *= s;
            else x /= s;
        }
        return *this;
    }

    template <typename S>
    image3d<T>& image_op (image3d<S> const& o, int op, char const* name)
    {
        if (dimx != o.dimx || dimy != o.dimy || dimz != o.dimz)
        {
            std::cout << "WARNING::image3d::operator" << name << " : dimensions must agree"
                      << std::endl;
            return *this;
        }
        for (size_t q = 0; q < rawimage.size(); ++q)
        {
            const T s = static_cast<T> (o.rawimage[q]);
            if (op == 0) rawimage[q] += s;
            else if (op == 1) rawimage[q] -= s;
            else if (op == 2) rawimage[q] *= s;
            else rawimage[q] /= s;
        }
        return *this;
    }
};

// binary operators copy the left operand, then apply the in-place one (:349-380)
template <typename S, typename R>
image3d<S> const operator+ (image3d<S> const& a, R const& b) { image3d<S> r (a); return r += b; }
template <typename S, typename R>
image3d<S> const operator- (image3d<S> const& a, R const& b) { image3d<S> r (a); return r -= b; }
template <typename S, typename R>
image3d<S> const operator* (image3d<S> const& a, R const& b) { image3d<S> r (a); return r *= b; }
template <typename S, typename R>
image3d<S> const operator/ (image3d<S> const& a, R const& b) { image3d<S> r (a); return r /= b; }

template <typename S, typename R>
S const scalarprod (image3d<S> const& a, image3d<R> const& b)
{
    if (a.dimx != b.dimx || a.dimy != b.dimy || a.dimz != b.dimz)
    {
        std::cout << "WARNING::scalarprod: dimensions must agree, 0 is returned" << std::endl;
        return 0;
    }
    S s = 0;
    for (size_t q = 0; q < a.rawimage.size(); ++q) s += a.rawimage[q] * static_cast<S> (b.rawimage[q]);
    return s;
}

template <typename S, typename R>
S const scalarprod_L2 (image3d<S> const& a, image3d<R> const& b)
{
    if (a.hx != b.hx || a.hy != b.hy || a.hz != b.hz)
    {
        std::cout << "WARNING::scalarprod_L2: spacing must agree, 0 is returned" << std::endl;
        return 0;
    }
    return a.hx * a.hy * a.hz * scalarprod (a, b);
}

template <typename S, typename R>
void vector_abs (image3d<S>& res, std::vector<image3d<R> > const& fun)
{
    if (fun.size() != 2 && fun.size() != 3)
    {
        std::cout << "In image3d::vector_abs: input vector could be only 2d or 3d, " << fun.size()
                  << " is a not allowed dimension." << std::endl;
        return;
    }
    res.setdim (fun[0].dimx, fun[0].dimy, fun[0].dimz);
    res.seth (fun[0].hx, fun[0].hy, fun[0].hz);
    for (size_t q = 0; q < res.rawimage.size(); ++q)
    {
        R s = 0;
        for (auto const& f : fun) s += f.rawimage[q] * f.rawimage[q];
        res.rawimage[q] = static_cast<S> (std::sqrt (s) );
    }
}

template <typename S, typename R>
void div (image3d<S>& res, std::vector<image3d<R> > const& fun)
{
    if (fun.size() != 3)
    {
        std::cout << "In image3d::div: input vector could be only 2d or 3d, " << fun.size()
                  << " is a not allowed dimension." << std::endl;
        return;
    }
    const uint X = fun[0].dimx, Y = fun[0].dimy, Z = fun[0].dimz;
    for (auto const& f : fun)
        if (f.dimx != X || f.dimy != Y || f.dimz != Z)
        {
            std::cout << "In image3d::div: dimensions of image3d inside input vector must agree"
                      << std::endl;
            return;
        }
    const size_t n = (size_t) X * Y * Z;
    std::vector<R> in (3 * n), out (n);
    for (int c = 0; c < 3; ++c) std::copy (fun[c].rawimage.begin(), fun[c].rawimage.end(), in.begin() + c * n);
    if (b200::failed (b200::ops<R>::div (b200::context(), in.data(), out.data(), X, Y, Z,
                                         fun[0].hx, fun[0].hy, fun[0].hz), "div") )
        return;
    res.setdim (X, Y, Z);
    res.seth (fun[0].hx, fun[0].hy, fun[0].hz);
    for (size_t q = 0; q < n; ++q) res.rawimage[q] = static_cast<S> (out[q]);
}

} // namespace im3d

#endif
