/*
 * poisson.hxx -- lapl::unsteady_poisson_functor<T>, lapl::DirGaussSeidel and
 * lapl::NeuGaussSeidel of the reference's header/poisson.hxx:54-195, on the B200
 * backend.
 *
 * One call is one in-place lexicographic sweep, exactly the reference's
 * (poisson_imp.hxx:340-429 and :23-336; bit for bit in double): the backend updates
 * the hyperplanes i+j+k = const in order, which gives every point the same new
 * minus-neighbours and old plus-neighbours as the reference's loops. RBGaussSeidel
 * (no counterpart in the reference) is one red-black sweep of the same equation.
 */
#ifndef IM3D_POISSON_HXX
#define IM3D_POISSON_HXX

#include "b200.hxx"
#include "image3d.hxx"

namespace lapl
{

template <typename T>
class unsteady_poisson_functor
{
private:
    void (*f) (im3d::image3d<T>& res, im3d::image3d<T> const& b, T const& dt, T const& bc,
               im3d::image3d<T> const& input);

public:
    unsteady_poisson_functor (void (*f) (im3d::image3d<T>& res, im3d::image3d<T> const& b,
                                         T const& dt, T const& bc, im3d::image3d<T> const& input) )
        : f (f)
    {
    }

    void operator() (im3d::image3d<T>& res, im3d::image3d<T> const& b, T const& dt = 1.,
                     T const& bc = 0., im3d::image3d<T> const& input = im3d::image3d<T>() )
    {
        this->f (res, b, dt, bc, input);
    }

    void changef (void (*f) (im3d::image3d<T>& res, im3d::image3d<T> const& b, T const& dt,
                             T const& bc, im3d::image3d<T> const& input) )
    {
        this->f = f;
    }

    auto function () const
        -> void (*) (im3d::image3d<T>&, im3d::image3d<T> const&, T const&, T const&,
                     im3d::image3d<T> const&)
    {
        return f;
    }
};

template <typename T>
void gpu_sweep (im3d::image3d<T>& res, im3d::image3d<T> const& b, T const& dt, T const& bc,
                int bc_type, int order, char const* who)
{
    im3d::b200::failed (im3d::b200::ops<T>::sweeps (im3d::b200::context(), res.data(), b.data(),
                                                    res.getdimx(), res.getdimy(), res.getdimz(),
                                                    res.gethx(), res.gethy(), res.gethz(), dt, bc,
                                                    bc_type, order, 1), who);
}

/* lapl::DirGaussSeidel: boundary := bc, one lexicographic sweep of the interior */
template <typename T>
void DirGaussSeidel (im3d::image3d<T>& res, im3d::image3d<T> const& b, T const& dt = 1.,
                     T const& bc = 0., im3d::image3d<T> const& input = im3d::image3d<T>() )
{
    (void) input;
    gpu_sweep (res, b, dt, bc, IM3D_BC_DIR, IM3D_SWEEP_LEXICOGRAPHIC, "DirGaussSeidel");
}

/* lapl::NeuGaussSeidel: outward normal derivative bc on the faces */
template <typename T>
void NeuGaussSeidel (im3d::image3d<T>& res, im3d::image3d<T> const& b, T const& dt = 1.,
                     T const& bc = 0., im3d::image3d<T> const& input = im3d::image3d<T>() )
{
    (void) input;
    gpu_sweep (res, b, dt, bc, IM3D_BC_NEU, IM3D_SWEEP_LEXICOGRAPHIC, "NeuGaussSeidel");
}

/* one red-black sweep with Dirichlet boundary (no counterpart in the reference) */
template <typename T>
void RBGaussSeidel (im3d::image3d<T>& res, im3d::image3d<T> const& b, T const& dt = 1.,
                    T const& bc = 0., im3d::image3d<T> const& input = im3d::image3d<T>() )
{
    (void) input;
    gpu_sweep (res, b, dt, bc, IM3D_BC_DIR, IM3D_SWEEP_REDBLACK, "RBGaussSeidel");
}

} // namespace lapl

#endif
