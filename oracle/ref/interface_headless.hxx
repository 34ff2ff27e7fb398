/*
 * interface_headless.hxx -- a headless stand-in for the reference's VTK-backed
 * im3d::interface<S> (header/interface.hxx:77-340), so that the reference's own
 * algorithm headers compile and run without VTK.
 *
 * TEST INFRASTRUCTURE ONLY: force-included (g++ -include) ahead of the reference
 * headers when oracle/Makefile builds the CPU checker. It defines the include
 * guard of the reference's interface.hxx first, so that the reference's
 * `#include "interface.hxx"` (image3d_imp.hxx:22) resolves to this class.
 *
 * Rendering (show_*) and picking (get_coordinates) are graphics paths with no
 * stack on this machine; they print one line and do nothing. The image is kept
 * as an image3d copy, and write() emits a MetaImage header plus raw doubles.
 */
#ifndef IM3D_ORACLE_INTERFACE_HEADLESS_HXX
#define IM3D_ORACLE_INTERFACE_HEADLESS_HXX

#define INTERFACE_HXX_INCLUDED
#define INTERFACE_IMP_HXX_INCLUDED
#define ABSTRACTINTERFACE_HXX_INCLUDED

#include "names.hxx"
#include "image3d.hxx"

#include <cstdio>
#include <string>

namespace im3d
{

template <typename S>
class interface
{
    image3d<S> stored;

public:
    interface () {}
    explicit interface (std::string const& imagename)
    {
        std::clog << "headless interface: reading " << imagename << " is not supported"
                  << std::endl;
    }
    explicit interface (image3d<S> const& myim) : stored (myim) {}
    virtual ~interface () {}

    void convertfromimage3d (image3d<S> const& myim) { this->stored = myim; }
    void convert2image3d (image3d<S>& myim) const { myim = this->stored; }

    void setcolour (double const& = 1., double const& = 1., double const& = 0.) {}
    void setopacity (double const& = 0.5) {}
    void show_contour (double const& = 0) {}
    void show_image () {}
    void show_image_and_contour (double const& = 0) {}
    void show_contour_with_background_image (interface&, double const& = 0) {}
    void get_coordinates (double& x, double& y, double& z) { x = y = z = 0; }
    void get_coordinates (uint& i, uint& j, uint& k) { i = j = k = 0; }
    void get_coordinates (double& x1, double& y1, double& z1,
                          double& x2, double& y2, double& z2)
    {
        x1 = y1 = z1 = x2 = y2 = z2 = 0;
    }
    void get_coordinates (uint& i1, uint& j1, uint& k1, uint& i2, uint& j2, uint& k2)
    {
        i1 = j1 = k1 = i2 = j2 = k2 = 0;
    }

    // MetaImage (.mhd + .raw, MET_DOUBLE, z-contiguous as image3d stores it)
    void write (std::string const& imagename = "image3d",
                std::string const& extension = "mhd") const
    {
        (void)extension;
        const uint X = stored.getdimx(), Y = stored.getdimy(), Z = stored.getdimz();
        std::string raw = imagename + ".raw";
        FILE* h = std::fopen ( (imagename + ".mhd").c_str(), "w");
        if (!h) return;
        std::fprintf (h, "ObjectType = Image\nNDims = 3\nBinaryData = True\n"
                      "BinaryDataByteOrderMSB = False\nDimSize = %u %u %u\n"
                      "ElementSpacing = %g %g %g\nElementType = MET_DOUBLE\n"
                      "ElementDataFile = %s\n", Z, Y, X,
                      stored.gethz(), stored.gethy(), stored.gethx(), raw.c_str() );
        std::fclose (h);
        FILE* r = std::fopen (raw.c_str(), "wb");
        if (!r) return;
        for (uint i = 0; i < X; ++i)
            for (uint j = 0; j < Y; ++j)
                for (uint k = 0; k < Z; ++k)
                {
                    double v = static_cast<double> (stored (i, j, k) );
                    std::fwrite (&v, sizeof (double), 1, r);
                }
        std::fclose (r);
    }
};

} // namespace im3d

#endif
