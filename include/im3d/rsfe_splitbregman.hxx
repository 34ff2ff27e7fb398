/*
 * rsfe_splitbregman.hxx -- segm::rsfe_splitbregman<T> of the reference
 * (header/rsfe_splitbregman.hxx:99-894, rsfe_splitbregman_imp.hxx) on the B200 backend.
 *
 * Same public members, defaults (imp :25-41), setter checks and WARNING texts
 * (imp :806-1440) and GetPot keys (imp :582-796). apply() runs the whole loop of
 * imp :1547-1995 on the GPU through im3d_rsfe_apply_*; phi is available afterwards
 * through getoutput().
 *
 * Plug-ins: the functors installed with set_cv / set_onestep_poisson / set_bc are
 * recognised and mapped onto the backend: acyclic_fftw_convolution and
 * direct_convolution (the same linear Gaussian filter), cyclic_fftw_convolution (the
 * periodic one), DirGaussSeidel,
 * NeuGaussSeidel (the reference's lexicographic sweep) and RBGaussSeidel (a red-black
 * sweep). Any other function pointer cannot run inside the GPU loop: apply() prints a
 * WARNING and uses the default of its kind.
 *
 * The automatic connected-component extraction (auto_extract_conn_comp with
 * auto_extract_conn_comp_freq and a cc_init_pixel seed, imp :448-536) runs on the GPU
 * inside the loop.
 *
 * dumpfrequency writes phi as "<outputname>_<t>" after every dumpfrequency-th iteration
 * but the last, and "<outputname>_<t>_final" at the end (imp :1940-1951, :1967-1979):
 * the loop hands phi to the host on those iterations only (im3d_ctx_set_observer).
 *
 * Not on this backend: interactive display (showfrequency, on-the-go updates) and the
 * interactive choice of a connected component, 2-D images.
 */
#ifndef IM3D_RSFE_SPLITBREGMAN_HXX
#define IM3D_RSFE_SPLITBREGMAN_HXX

#include <algorithm>
#include <cstdio>
#include <sstream>
#include <string>

#include "b200.hxx"
#include "convolution.hxx"
#include "getpot.hxx"
#include "image3d.hxx"
#include "poisson.hxx"
#include "segmentation.hxx"

namespace segm
{

template <typename T>
class rsfe_splitbregman : public segmentation<T>
{
private:
    enum bc_type { NEU = 1, DIR };
    enum ed_type { GRAD = 1, GRAD_THRESHOLD, LBP };

    std::string getpotfile = "data";
    bool verbosity = true;
    uint maxiter = 100;
    uint showfrequency = 0;
    uint dumpfrequency = 0;
    std::string outputname = "result";
    std::string logfilename = "";
    bool onthego = true;
    bool save_current = false;
    bool end_now = false;
    T sigma = 3, lamda = 5.e-2, lamda1 = 1.e-5, lamda2 = 1.e-5, beta = 100., dt = 1;
    uint ls_steps = 5;
    T epsilon = 1.e-3, a0 = 0., b0 = 1.;
    bool auto_extract_conn_comp = false;
    double cc_init_pixel_x = -1, cc_init_pixel_y = -1, cc_init_pixel_z = -1;
    bool cc_binary_output = true, cc_init_variables = true;
    uint auto_extract_conn_comp_freq = 0;
    bc_type bc = NEU;
    T ls_tol = 0;
    ed_type edge_detector = GRAD;
    T edge_detector_sigma = 0;
    T nu = 1.;
    lapl::unsteady_poisson_functor<T> onestep_poisson {lapl::DirGaussSeidel<T>};
    conv::filtering<T> cv {conv::acyclic_fftw_convolution<T>};
    bool gaussian_pixel_approach = false;
    T tol = 1.e-5;
    int ix = -1, iy = -1, iz = -1, fx = -1, fy = -1, fz = -1;
    uint dimx = 0, dimy = 0, dimz = 1;
    bool init_variables = false;
    // backend extensions
    double gs_rel_res_tol = 0, omega = 1;
    int gs_max_sweeps = 1000;
    im3d_rsfe_stats last_stats {};

    void say (std::string const& k, double v) const
    {
        if (verbosity) std::clog << "---\t" << k << " = " << v << std::endl;
    }

    void set_param_from_getpot (std::string const& section)
    {
        im3d::getpot_file f (getpotfile.c_str(), "#");
        f.set_prefix ( ("splitbregman/" + section).c_str() );
        int it;
        double d;
        std::string s;
        if ( (it = f ("verbosity", -1) ) != -1) set_verbosity (it != 0);
        if ( (it = f ("maxiter", -1) ) > 0) set_maxiter (it);
        if ( (it = f ("showfrequency", -1) ) >= 0) set_showfrequency (it);
        if ( (it = f ("dumpfrequency", -1) ) >= 0) set_dumpfrequency (it);
        if ( (s = f ("outputname", "") ).size() != 0) set_outputname (s);
        if ( (it = f ("save_current", -1) ) != -1) save_current = it != 0;
        if ( (it = f ("end_now", -1) ) != -1) end_now = it != 0;
        if ( (d = f ("sigma", -1.) ) != -1.) set_sigma (d);
        if ( (d = f ("lamda", -1.) ) != -1.) set_lamda (d);
        if ( (d = f ("lamda1", -1.) ) != -1.) set_lamda1 (d);
        if ( (d = f ("lamda2", -1.) ) != -1.) set_lamda2 (d);
        if ( (d = f ("nu", -1.) ) != -1.) set_nu (d);
        if ( (d = f ("beta", -1.) ) != -1.) set_beta (d);
        if ( (d = f ("dt", -1.) ) != -1.) set_dt (d);
        if ( (it = f ("ls_steps", -1) ) != -1) set_ls_steps ( (uint) it);
        if ( (d = f ("epsilon", -1.) ) != -1.) set_epsilon (d);
        if ( (d = f ("a0", 2.1e-6) ) != 2.1e-6) set_a0 (d);
        if ( (d = f ("b0", -2.1e-6) ) != -2.1e-6) set_b0 (d);
        if ( (it = f ("auto_extract_conn_comp", -1) ) != -1) set_auto_extract_conn_comp (it != 0);
        if ( (it = f ("cc_binary_output", -1) ) != -1) set_cc_binary_output (it != 0);
        if ( (it = f ("cc_init_variables", -1) ) != -1) set_cc_init_variables (it != 0);
        if ( (d = f ("cc_init_pixel_x", -1.) ) != -1.) set_cc_init_pixel_x (d);
        if ( (d = f ("cc_init_pixel_y", -1.) ) != -1.) set_cc_init_pixel_y (d);
        if ( (d = f ("cc_init_pixel_z", -1.) ) != -1.) set_cc_init_pixel_z (d);
        if ( (it = f ("auto_extract_conn_comp_freq", -1) ) >= 0) set_auto_extract_conn_comp_freq (it);
        if ( (it = f ("bc", -1) ) != -1) set_bc (static_cast<bc_type> (it) );
        if ( (d = f ("ls_tol", -1.) ) != -1.) set_ls_tol (d);
        if ( (it = f ("edge_detector", -1) ) != -1) set_edge_detector (static_cast<ed_type> (it) );
        if ( (d = f ("edge_detector_sigma", -1.) ) != -1.) set_edge_detector_sigma (d);
        if ( (it = f ("gaussian_pixel_approach", -1) ) != -1) set_gaussian_pixel_approach (it != 0);
        if ( (d = f ("tol", -1.) ) != -1.) set_tol (d);
        if ( (d = f ("alpha", 1.e-9) ) != 1.e-9) set_alpha (d);
    }

    // the initial level set of initialize_phi_with_init (imp :99-170): same size, or
    // one voxel smaller per axis (last face repeated); otherwise the default cube
    bool expand_init (im3d::image3d<T> const& init, std::vector<T>& out) const
    {
        const uint X = init.getdimx(), Y = init.getdimy(), Z = init.getdimz();
        if (! ( (X == dimx || X + 1 == dimx) && (Y == dimy || Y + 1 == dimy) &&
                (Z == dimz || Z + 1 == dimz) ) )
        {
            std::clog << "WARNING::apply: wrong dimensions of init, cube initial "
                      << "contour is used instead." << std::endl;
            return false;
        }
        out.assign ( (size_t) dimx * dimy * dimz, T (0) );
        for (uint i = 0; i < dimx; ++i)
            for (uint j = 0; j < dimy; ++j)
                for (uint k = 0; k < dimz; ++k)
                    out[ ( (size_t) i * dimy + j) * dimz + k] =
                        init (i < X ? i : X - 1, j < Y ? j : Y - 1, k < Z ? k : Z - 1);
        return true;
    }

    int backend_bc () const
    {
        auto f = onestep_poisson.function();
        if (f == &lapl::NeuGaussSeidel<T>)
        {
            if (bc != NEU)
                std::clog << "WARNING::apply: NeuGaussSeidel with bc = DIR is not on the B200 "
                          << "backend, flux 0 is used" << std::endl;
            return IM3D_BC_NEU;
        }
        if (f != &lapl::DirGaussSeidel<T> && f != &lapl::RBGaussSeidel<T>)
            std::clog << "WARNING::apply: custom Poisson step not supported by the B200 "
                      << "backend, DirGaussSeidel is used" << std::endl;
        return bc == DIR ? IM3D_BC_DIR : IM3D_BC_DEFAULT;
    }

public:
    rsfe_splitbregman () : segmentation<T>() { this->alpha = (this->a0 + this->b0) / 2.; }

    // ---- members not settable from the GetPot file (imp :806-852)
    inline void set_getpotfile (std::string const& name) { getpotfile = name; }
    inline void set_onthego (bool const o) { onthego = o; }
    inline void set_logfilename (std::string const& name) { logfilename = name; }
    inline void set_cv (conv::filtering<T> const c) { cv = c; }
    inline void set_onestep_poisson (lapl::unsteady_poisson_functor<T> const osl) { onestep_poisson = osl; }

    // ---- members settable from the GetPot file (imp :857-1440)
    inline void set_verbosity (bool const v)
    {
        verbosity = v;
        if (verbosity) std::clog << "---\tverbosity = " << verbosity << std::endl;
    }
    inline void set_maxiter (uint const& m) { maxiter = m; say ("maxiter", m); }
    inline void set_showfrequency (uint const& s) { showfrequency = s; say ("showfrequency", s); }
    inline void set_auto_extract_conn_comp_freq (uint const& c) { auto_extract_conn_comp_freq = c; say ("auto_extract_conn_comp_freq", c); }
    inline void set_dumpfrequency (uint const& d) { dumpfrequency = d; say ("dumpfrequency", d); }
    inline void set_outputname (std::string const& name)
    {
        outputname = name;
        if (verbosity) std::clog << "---\toutputname = " << outputname << std::endl;
    }
    inline void set_tol (T const& t)
    {
        if (t >= 0) { tol = t; say ("tol", t); }
        else std::clog << "WARNING::set_tol: tol must be greater than zero" << std::endl;
    }
    inline void set_cc_init_pixel_x (double const& v)
    {
        if (v >= 0) { cc_init_pixel_x = v; say ("cc_init_pixel_x", v); }
        else std::clog << "WARNING::set_cc_init_pixel_x: coordinates must be positive" << std::endl;
    }
    inline void set_cc_init_pixel_y (double const& v)
    {
        if (v >= 0) { cc_init_pixel_y = v; say ("cc_init_pixel_y", v); }
        else std::clog << "WARNING::set_cc_init_pixel_y: coordinates must be positive" << std::endl;
    }
    inline void set_cc_init_pixel_z (double const& v)
    {
        if (v >= 0) { cc_init_pixel_z = v; say ("cc_init_pixel_z", v); }
        else std::clog << "WARNING::set_cc_init_pixel_z: coordinates must be positive" << std::endl;
    }
    inline void set_lamda (T const& v)
    {
        if (v > 0) { lamda = v; say ("lamda", v); }
        else std::clog << "WARNING::set_lamda: lamda must be greater than zero" << std::endl;
    }
    inline void set_lamda1 (T const& v)
    {
        if (v > 0) { lamda1 = v; say ("lamda1", v); }
        else std::clog << "WARNING::set_lamda1: lamda1 must be greater than zero" << std::endl;
    }
    inline void set_lamda2 (T const& v)
    {
        if (v > 0) { lamda2 = v; say ("lamda2", v); }
        else std::clog << "WARNING::set_lamda2: lamda2 must be greater than zero" << std::endl;
    }
    inline void set_sigma (T const& v)
    {
        if (v > 0) { sigma = v; say ("sigma", v); }
        else std::clog << "WARNING::set_sigma: sigma must be greater than zero" << std::endl;
    }
    inline void set_edge_detector_sigma (T const& v)
    {
        if (v >= 0) { edge_detector_sigma = v; say ("edge_detector_sigma", v); }
        else std::clog << "WARNING::set_edge_detector_sigma: edge_detector_sigma must be greater than zero" << std::endl;
    }
    inline void set_nu (T const& v)
    {
        if (v >= 0) { nu = v; say ("nu", v); }
        else std::clog << "WARNING::set_nu: nu must be non negative" << std::endl;
    }
    inline void set_beta (T const& v)
    {
        if (v >= 0) { beta = v; say ("beta", v); }
        else std::clog << "WARNING::set_beta: beta must be non negative" << std::endl;
    }
    inline void set_dt (T const& v)
    {
        if (v > 0) { dt = v; say ("dt", v); }
        else std::clog << "WARNING::set_dt: dt must be greater than zero" << std::endl;
    }
    inline void set_a0 (T const& v)
    {
        a0 = v;
        this->alpha = (a0 + b0) / 2.;
        say ("a0", a0);
        say ("  alpha", this->alpha);
        if (b0 < a0)
        {
            b0 = a0 + 1;
            this->alpha = (a0 + b0) / 2.;
            std::clog << "WARNING::set_a0: b0 has to be greater than a0, hence its value is "
                      << "automatically modified" << std::endl;
            std::clog << "---\t  b0 = " << b0 << std::endl << "---\t  alpha = " << this->alpha << std::endl;
        }
    }
    inline void set_b0 (T const& v)
    {
        b0 = v;
        this->alpha = (a0 + b0) / 2.;
        say ("b0", b0);
        say ("  alpha", this->alpha);
        if (b0 < a0)
        {
            a0 = b0 - 1;
            this->alpha = (a0 + b0) / 2.;
            std::clog << "WARNING::set_b0: a0 has to be lower than b0, hence its value is "
                      << "automatically modified" << std::endl;
            std::clog << "---\t  a0 = " << a0 << std::endl << "---\t  alpha = " << this->alpha << std::endl;
        }
    }
    inline void set_epsilon (T const& v)
    {
        if (v > 0) { epsilon = v; say ("epsilon", v); }
        else std::clog << "WARNING::set_epsilon: epsilon must be greater than zero" << std::endl;
    }
    inline void set_bc (bc_type const b)
    {
        if (b == NEU)
        {
            bc = b;
            onestep_poisson.changef (lapl::NeuGaussSeidel<T>);
            if (verbosity) std::clog << "---\tbc = NEU" << std::endl;
        }
        else if (b == DIR)
        {
            bc = b;
            onestep_poisson.changef (lapl::DirGaussSeidel<T>);
            if (verbosity) std::clog << "---\tbc = DIR" << std::endl;
        }
        else
        {
            std::clog << "WARNING::set_bc: specify a proper bc_type condition" << std::endl;
        }
    }
    inline void set_ls_tol (T const& v)
    {
        if (v >= 0) { ls_tol = v; say ("ls_tol", v); }
        else std::clog << "WARNING::set_tol: tol must be positive" << std::endl;
    }
    inline void set_ls_steps (uint const s)
    {
        if (s > 0) { ls_steps = s; say ("ls_steps", s); }
        else std::clog << "WARNING::set_ls_steps: ls_steps must be greater than 0" << std::endl;
    }
    inline void set_gaussian_pixel_approach (bool const g) { gaussian_pixel_approach = g; }
    inline void set_edge_detector (ed_type const e)
    {
        if (e == 1 || e == 2 || e == 3) edge_detector = e;
        else std::clog << "WARNING::set_edge_detector: specify a proper ed_type condition" << std::endl;
    }
    inline void set_auto_extract_conn_comp (bool const a) { auto_extract_conn_comp = a; say ("auto_extract_conn_comp", a); }
    inline void set_cc_binary_output (bool const c) { cc_binary_output = c; say ("cc_binary_output", c); }
    inline void set_cc_init_variables (bool const c) { cc_init_variables = c; say ("cc_init_variables", c); }
    inline void set_alpha (T const& a)
    {
        if (a > a0 && a < b0) { this->alpha = a; say ("alpha", a); }
        else std::clog << "WARNING::set_alpha: alpha must be greater than a0 and less than b0" << std::endl;
    }

    // ---- backend extensions (no counterpart in the reference)
    /* > 0: each outer iteration solves (1/dt - Lap) u = u_old/dt + rhs to this relative
     * residual with red-black sweeps, instead of ls_steps reference sweeps */
    inline void set_gs_rel_res_tol (double t) { gs_rel_res_tol = t > 0 ? t : 0; }
    inline void set_omega (double w) { omega = w; }
    inline void set_gs_max_sweeps (int m) { gs_max_sweeps = m; }
    inline im3d_rsfe_stats const& get_stats () const { return last_stats; }

    // ---- the algorithm
    void apply (im3d::image3d<T> const& myim) { run (myim, nullptr); }

    void apply (im3d::image3d<T> const& myim, im3d::image3d<T> const& init) { run (myim, &init); }

private:
    // the dump of imp :1940-1951, called by the GPU loop with a host copy of phi
    static int dump_observer (void* user, im3d_rsfe_checkpoint const* ck)
    {
        rsfe_splitbregman* self = static_cast<rsfe_splitbregman*> (user);
        T const* src = static_cast<T const*> (ck->phi);
        std::copy (src, src + (size_t) self->dimx * self->dimy * self->dimz, self->phi.data() );
        self->levelset.convertfromimage3d (self->phi);
        std::ostringstream oss;
        oss << self->outputname << "_" << ck->t;
        self->levelset.write (oss.str() );
        return 0;
    }

    void run (im3d::image3d<T> const& myim, im3d::image3d<T> const* init)
    {
        FILE* redirected = nullptr;
        if (logfilename != "") redirected = std::freopen (logfilename.c_str(), "a", stderr);
        std::clog << "- RSFE/Split-Bregman Algorithm for 3d image segmentation" << std::endl;
        if (getpotfile != "")
        {
            if (verbosity)
                std::clog << "-- Initializing parameters of algorithm from file " << getpotfile
                          << " (section splitbregman/init/)" << std::endl;
            set_param_from_getpot ("init/");
        }
        else
        {
            onthego = false;
        }
        dimx = myim.getdimx();
        dimy = myim.getdimy();
        dimz = myim.getdimz();
        std::clog << "- Sizeof(phi): " << sizeof (T) * dimx * dimy * dimz << " byte" << std::endl;
        std::clog << "- dimensions:\t" << dimx << " x " << dimy << " x " << dimz << std::endl;
        std::clog << "- spacing:\t" << myim.gethx() << " x " << myim.gethy() << " x "
                  << myim.gethz() << std::endl;
        if (showfrequency)
            std::clog << "WARNING::apply: display (and the interactive connected-component "
                      << "choice) is not part of the B200 backend" << std::endl;
        auto cvf = cv.function();
        if (cvf != &conv::acyclic_fftw_convolution<T> && cvf != &conv::direct_convolution<T> &&
                cvf != &conv::cyclic_fftw_convolution<T>)
            std::clog << "WARNING::apply: custom convolution not supported by the B200 backend, "
                      << "the Gaussian filter is used" << std::endl;

        im3d_rsfe_params p;
        im3d_rsfe_params_default (&p);
        p.tol = tol;
        p.sigma = sigma;
        p.lamda = lamda;
        p.lamda1 = lamda1;
        p.lamda2 = lamda2;
        p.beta = beta;
        p.nu = nu;
        p.dt = dt;
        p.epsilon = epsilon;
        p.a0 = a0;
        p.b0 = b0;
        p.ls_tol = ls_tol;
        p.edge_detector_sigma = edge_detector_sigma;
        p.maxiter = (int32_t) maxiter;
        p.ls_steps = (int32_t) ls_steps;
        p.bc = backend_bc();
        p.gaussian_pixel_approach = gaussian_pixel_approach ? 1 : 0;
        p.init_variables = init_variables ? 1 : 0;
        p.sweep = onestep_poisson.function() == &lapl::RBGaussSeidel<T> ? IM3D_SWEEP_REDBLACK
                                                                          : IM3D_SWEEP_LEXICOGRAPHIC;
        p.gs_rel_res_tol = gs_rel_res_tol;
        p.omega = omega;
        p.gs_max_sweeps = gs_max_sweeps;
        p.alpha = this->alpha;
        p.auto_extract_conn_comp = auto_extract_conn_comp ? 1 : 0;
        p.auto_extract_conn_comp_freq = (int32_t) auto_extract_conn_comp_freq;
        p.cc_init_pixel_x = cc_init_pixel_x;
        p.cc_init_pixel_y = cc_init_pixel_y;
        p.cc_init_pixel_z = cc_init_pixel_z;
        p.cc_binary_output = cc_binary_output ? 1 : 0;
        p.cc_init_variables = cc_init_variables ? 1 : 0;
        p.conv_cyclic = cvf == &conv::cyclic_fftw_convolution<T> ? 1 : 0;

        std::vector<T> full;
        T const* ini = nullptr;
        if (init && expand_init (*init, full) ) ini = full.data();

        this->phi.setdim (dimx, dimy, dimz);
        this->phi.seth (myim.gethx(), myim.gethy(), myim.gethz() );
        im3d_ctx* bctx = im3d::b200::context();
        if (bctx && dumpfrequency > 0)
            im3d_ctx_set_observer (bctx, (int) dumpfrequency, 0, &rsfe_splitbregman::dump_observer, this);
        const int st = im3d::b200::ops<T>::apply (bctx, myim.data(), ini, dimx, dimy,
                                                  dimz, myim.gethx(), myim.gethy(), myim.gethz(), &p,
                                                  this->phi.data(), &last_stats);
        if (bctx && dumpfrequency > 0) im3d_ctx_set_observer (bctx, 0, 0, nullptr, nullptr);
        if (!im3d::b200::failed (st, "apply") )
        {
            if (verbosity)
                std::clog << "-- " << last_stats.iterations << " iterations, norm_L2: "
                          << last_stats.last_tol << ", sweeps: " << last_stats.total_sweeps << std::endl;
            this->levelset.convertfromimage3d (this->phi);
            this->image.convertfromimage3d (myim);
            if (dumpfrequency > 0)
            {
                std::ostringstream oss;
                oss << outputname << "_" << last_stats.iterations << "_final";
                this->levelset.write (oss.str() );
            }
        }
        ix = iy = iz = fx = fy = fz = -1;
        if (redirected) std::fclose (stderr);
    }
};

} // namespace segm

#endif
