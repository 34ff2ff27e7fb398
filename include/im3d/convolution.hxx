/*
 * convolution.hxx -- conv::filtering<T> and the convolution functions of the
 * reference's header/convolution.hxx:72-411, on the B200 backend.
 *
 * build_gaussian_filter keeps the Gaussian's parameters (and, as the reference does,
 * its time-domain samples in the public static time_filter); acyclic_fftw_convolution
 * and direct_convolution then filter on the GPU (im3d_gauss_filter_*). Both are the
 * same linear convolution with zero boundary in the reference
 * (convolution_imp.hxx:535-653 and :761-812); the backend evaluates it as three 1-D
 * passes of the normalised Gaussian. cyclic_fftw_convolution (:657-754) takes the
 * volume as periodic and runs as the same passes with wrapped indices
 * (im3d_gauss_filter_cyclic_*). Filters other than the Gaussian
 * (build_high_pass_filter, build_laplacian_filter) are not part of this backend.
 */
#ifndef IM3D_CONVOLUTION_HXX
#define IM3D_CONVOLUTION_HXX

#include <cmath>

#include "b200.hxx"
#include "image3d.hxx"

namespace conv
{

template <typename T>
class filtering
{
private:
    void (*f) (im3d::image3d<T>& result, im3d::image3d<T> const& factor);

public:
    filtering (void (*f) (im3d::image3d<T>& result, im3d::image3d<T> const& factor) ) : f (f) {}

    void operator() (im3d::image3d<T>& result, im3d::image3d<T> const& factor) const
    {
        this->f (result, factor);
    }

    void changef (void (*newf) (im3d::image3d<T>& result, im3d::image3d<T> const& factor) )
    {
        this->f = newf;
    }

    // the function currently installed (used by rsfe_splitbregman to recognise it)
    auto function () const -> void (*) (im3d::image3d<T>&, im3d::image3d<T> const&) { return f; }

    static im3d::image3d<T> time_filter;

    // parameters of the last build_gaussian_filter
    static double sigma;
    static double radius;
    static bool pixel_approach;
    static bool built;

    /* convolution_imp.hxx:22-91: Nh = odd(ceil(2 radius sigma / h)) samples per axis of
     * exp(-|d|^2 / (2 sigma^2)), normalised to unit L1 norm. */
    static void build_gaussian_filter (im3d::image3d<T> const& f, T const& sigma,
                                       double const& radius = 3, bool pixel_approach = false)
    {
        double hx = f.gethx(), hy = f.gethy(), hz = f.gethz();
        if (pixel_approach) hx = hy = hz = 1.;
        int nx = (int) std::ceil (2 * radius * sigma / hx);
        int ny = (int) std::ceil (2 * radius * sigma / hy);
        int nz = f.getdimz() == 1 ? 1 : (int) std::ceil (2 * radius * sigma / hz);
        nx += (nx % 2 == 0);
        ny += (ny % 2 == 0);
        nz += (nz % 2 == 0);
        time_filter.setdim (nx, ny, nz);
        time_filter.seth (f.gethx(), f.gethy(), f.gethz() );
        const int sx = nx / 2, sy = ny / 2, sz = nz / 2;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k)
                    time_filter (i, j, k) =
                        std::exp ( (- (i - sx) * (i - sx) * hx * hx - (j - sy) * (j - sy) * hy * hy -
                                    (k - sz) * (k - sz) * hz * hz) / (2 * sigma * sigma) );
        time_filter /= time_filter.normL1();
        filtering<T>::sigma = sigma;
        filtering<T>::radius = radius;
        filtering<T>::pixel_approach = pixel_approach;
        filtering<T>::built = true;
    }

    /* The GPU filters from the stored parameters; nothing to precompute per size. */
    static void build_freq_filters (im3d::image3d<T> const& f) { (void) f; }
};

template <typename T> im3d::image3d<T> filtering<T>::time_filter;
template <typename T> double filtering<T>::sigma = 0;
template <typename T> double filtering<T>::radius = 3;
template <typename T> bool filtering<T>::pixel_approach = false;
template <typename T> bool filtering<T>::built = false;

template <typename T>
void gaussian_gpu_filter (im3d::image3d<T>& result, im3d::image3d<T> const& factor, char const* who,
                          bool cyclic = false)
{
    if (!filtering<T>::built)
    {
        std::clog << "WARNING::" << who << ": build_gaussian_filter has not been called" << std::endl;
        return;
    }
    if (result.getdimx() != factor.getdimx() || result.getdimy() != factor.getdimy() ||
            result.getdimz() != factor.getdimz() )
        result.setdim (factor.getdimx(), factor.getdimy(), factor.getdimz() );
    result.seth (factor.gethx(), factor.gethy(), factor.gethz() );
    im3d::b200::failed (im3d::b200::ops<T>::gauss (im3d::b200::context(), factor.data(), result.data(),
                                                   factor.getdimx(), factor.getdimy(), factor.getdimz(),
                                                   factor.gethx(), factor.gethy(), factor.gethz(),
                                                   filtering<T>::sigma, filtering<T>::radius,
                                                   filtering<T>::pixel_approach ? 1 : 0, cyclic ? 1 : 0),
                        who);
}

/* conv::acyclic_fftw_convolution (convolution_imp.hxx:535-653) */
template <typename T>
void acyclic_fftw_convolution (im3d::image3d<T>& result, im3d::image3d<T> const& factor)
{
    gaussian_gpu_filter (result, factor, "acyclic_fftw_convolution");
}

/* conv::cyclic_fftw_convolution (convolution_imp.hxx:657-754): periodic boundary */
template <typename T>
void cyclic_fftw_convolution (im3d::image3d<T>& result, im3d::image3d<T> const& factor)
{
    gaussian_gpu_filter (result, factor, "cyclic_fftw_convolution", true);
}

/* conv::direct_convolution (convolution_imp.hxx:761-812): the same linear convolution */
template <typename T>
void direct_convolution (im3d::image3d<T>& result, im3d::image3d<T> const& factor)
{
    gaussian_gpu_filter (result, factor, "direct_convolution");
}

} // namespace conv

#endif
