// Checks of the header-only C++ API (include/im3d/) against the reference's known
// answers (examples/test.cxx) and writes GPU results for the pytest driver
// (tests/test_cpp_api.py) to compare with the CPU checker.
//
//   api_check <workdir>
//
// Prints one "ok <name>" / "FAIL <name> ..." line per check, exits non-zero on failure.
#include <cmath>
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "im3d/convolution.hxx"
#include "im3d/image3d.hxx"
#include "im3d/interface.hxx"
#include "im3d/poisson.hxx"
#include "im3d/rsfe_splitbregman.hxx"

static int failures = 0;

static void check (bool ok, std::string const& name, double got = 0, double want = 0)
{
    if (ok) std::cout << "ok " << name << std::endl;
    else
    {
        std::cout << "FAIL " << name << " got " << got << " want " << want << std::endl;
        ++failures;
    }
}

static bool all_equal (im3d::image3d<double> const& a, double v)
{
    for (size_t q = 0; q < a.size(); ++q)
        if (a.data() [q] != v) return false;
    return true;
}

int main (int argc, char** argv)
{
    const std::string dir = argc > 1 ? argv[1] : ".";
    // examples/test.cxx:101-201: operators and scalar products
    im3d::image3d<double> a (3, 3, 3), b (3, 3, 3), c;
    a = 1.5;
    b = a;
    a += b;
    check (all_equal (a, 3.), "operator+=");
    a -= b;
    check (all_equal (a, 1.5), "operator-=");
    a *= b;
    check (all_equal (a, 2.25), "operator*=");
    a /= b;
    check (all_equal (a, 1.5), "operator/=");
    c = a + b;
    check (all_equal (c, 3.), "operator+");
    c = a / 1.5;
    check (all_equal (c, 1.), "operator/");
    c = 1.;
    check (im3d::scalarprod (a, c) == 40.5, "scalarprod", im3d::scalarprod (a, c), 40.5);
    check (im3d::scalarprod_L2 (a, c) == 40.5, "scalarprod_L2");
    im3d::image3d<double> small (2, 2, 2);
    a += small;  // mismatch: WARNING, unchanged
    check (all_equal (a, 1.5), "mismatch_leaves_operand");

    // examples/test.cxx:226-252: grad of enumerate, div(grad), norms
    im3d::image3d<double> e (3, 3, 3);
    for (uint k = 0; k < 3; ++k)
        for (uint j = 0; j < 3; ++j)
            for (uint i = 0; i < 3; ++i) e (i, j, k) = i + 3 * j + 9 * k;
    std::vector<im3d::image3d<double> > g;
    e.grad (g);
    check (g.size() == 3 && all_equal (g[0], 1) && all_equal (g[1], 3) && all_equal (g[2], 9),
           "grad_enumerate");
    im3d::image3d<double> dv;
    im3d::div (dv, g);
    check (all_equal (dv, 0), "div_grad");
    check (e.norm1() == 351 && e.normL1() == 351, "norm1", e.norm1(), 351);
    check (e.norminf() == 26 && e.max() == 26 && e.min() == 0, "norminf_max_min");

    // Gaussian filter and a Gauss-Seidel sweep on a read volume
    im3d::interface<double> rd;
    if (!rd.load (dir + "/vol.mhd") ) { std::cout << "FAIL read" << std::endl; return 2; }
    im3d::image3d<double> u0;
    rd.convert2image3d (u0);
    conv::filtering<double> f (conv::acyclic_fftw_convolution<double>);
    conv::filtering<double>::build_gaussian_filter (u0, 2.0);
    im3d::image3d<double> fu;
    f (fu, u0);
    im3d::interface<double> (fu).write (dir + "/conv_out");
    im3d::image3d<double> r (u0), rhs (u0);
    rhs *= 0.5;
    lapl::unsteady_poisson_functor<double> gs (lapl::DirGaussSeidel<double>);
    gs (r, rhs, 0.7, 0.25);
    gs (r, rhs, 0.7, 0.25);
    im3d::interface<double> (r).write (dir + "/gs_out");

    // the segmentation class with a GetPot file
    segm::rsfe_splitbregman<double> algo;
    algo.set_verbosity (false);
    algo.set_getpotfile (dir + "/params.pot");
    im3d::interface<double> ri;
    if (!ri.load (dir + "/init.mhd") ) { std::cout << "FAIL read init" << std::endl; return 2; }
    im3d::image3d<double> init;
    ri.convert2image3d (init);
    algo.apply (u0, init);
    im3d::interface<double> (algo.getoutput() ).write (dir + "/phi_out");
    std::cout << "iterations " << algo.get_stats().iterations << std::endl;

    // connected component of the read volume, and black & white conversion
    im3d::image3d<double> cc, bw;
    u0.connected_component (cc, 10, 9, 8, 0.5, true);
    im3d::interface<double> (cc).write (dir + "/cc_out");
    u0.im_to_black_and_white (bw, 0.5);
    const double pivot = u0.min() + (u0.max() - u0.min() ) * 0.5;
    bool bw_ok = true;
    for (size_t q = 0; q < bw.size(); ++q)
        bw_ok = bw_ok && bw.data() [q] == (u0.data() [q] < pivot ? 0. : 1.);
    check (bw_ok, "im_to_black_and_white");

    // the loop with the automatic connected-component extraction
    segm::rsfe_splitbregman<double> algo2;
    algo2.set_verbosity (false);
    algo2.set_getpotfile (dir + "/params.pot");
    algo2.set_auto_extract_conn_comp (true);
    algo2.set_auto_extract_conn_comp_freq (2);
    algo2.set_cc_init_pixel_x (10);
    algo2.set_cc_init_pixel_y (9);
    algo2.set_cc_init_pixel_z (8);
    algo2.apply (u0, init);
    im3d::interface<double> (algo2.getoutput() ).write (dir + "/phi_cc_out");
    return failures ? 1 : 0;
}
