/*
 * interface.hxx -- im3d::interface<S>, the headless counterpart of the reference's
 * VTK-backed class (header/interface.hxx:77-340, abstractinterface.hxx:45-169).
 *
 * Kept: reading and writing MetaImage volumes (.mhd header + raw data; the reference
 * reads them through vtkMetaImageReader, interface_imp.hxx:34-90, and writes them
 * through vtkMetaImageWriter, :672-712), and the conversions to and from image3d.
 * Not available here: rendering, contour display and picking (show_*,
 * get_coordinates), which need a graphics stack; those members print one line and
 * leave their arguments unchanged. DICOM, JPEG and BMP readers are not part of this
 * backend.
 *
 * MetaImage axis order: DimSize lists the fastest axis first. image3d's fastest axis
 * is k, so DimSize = dimz dimy dimx and ElementSpacing = hz hy hx.
 */
#ifndef IM3D_INTERFACE_HXX
#define IM3D_INTERFACE_HXX

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "image3d.hxx"

namespace im3d
{

template <typename S>
class interface
{
    image3d<S> stored;

    static std::string trim (std::string const& s)
    {
        size_t a = s.find_first_not_of (" \t\r\n");
        if (a == std::string::npos) return "";
        size_t b = s.find_last_not_of (" \t\r\n");
        return s.substr (a, b - a + 1);
    }

    template <typename E>
    static void read_raw (std::ifstream& f, size_t n, std::vector<double>& out)
    {
        std::vector<E> buf (n);
        f.read (reinterpret_cast<char*> (buf.data() ), (std::streamsize) (n * sizeof (E) ) );
        out.resize (n);
        for (size_t q = 0; q < n; ++q) out[q] = static_cast<double> (buf[q]);
    }

public:
    interface () {}
    explicit interface (std::string const& imagename) { this->load (imagename); }
    explicit interface (image3d<S> const& myim) : stored (myim) {}
    virtual ~interface () {}

    /* MetaImage reader (.mhd with ElementDataFile, or .mha with LOCAL data). Element
     * types MET_UCHAR, MET_CHAR, MET_USHORT, MET_SHORT, MET_UINT, MET_INT, MET_FLOAT,
     * MET_DOUBLE, little endian. Returns false (with a WARNING) on failure. */
    bool load (std::string const& name)
    {
        std::ifstream h (name, std::ios::binary);
        if (!h)
        {
            std::clog << "WARNING::interface: cannot open " << name << std::endl;
            return false;
        }
        int ndims = 3;
        std::vector<long> dims;
        std::vector<double> sp (3, 1.0);
        std::string type, datafile;
        bool msb = false;
        std::string line;
        std::streampos data_pos = 0;
        while (std::getline (h, line) )
        {
            size_t eq = line.find ('=');
            if (eq == std::string::npos) continue;
            std::string key = trim (line.substr (0, eq) ), val = trim (line.substr (eq + 1) );
            std::istringstream vs (val);
            if (key == "NDims") vs >> ndims;
            else if (key == "DimSize") { long v; while (vs >> v) dims.push_back (v); }
            else if (key == "ElementSpacing" || key == "ElementSize") { sp.clear(); double v; while (vs >> v) sp.push_back (v); }
            else if (key == "ElementType") type = val;
            else if (key == "BinaryDataByteOrderMSB" || key == "ElementByteOrderMSB") msb = (val == "True");
            else if (key == "ElementDataFile")
            {
                datafile = val;
                data_pos = h.tellg();
                break;
            }
        }
        if (msb || dims.empty() || ndims < 2 || ndims > 3)
        {
            std::clog << "WARNING::interface: unsupported MetaImage header in " << name << std::endl;
            return false;
        }
        while (dims.size() < 3) dims.push_back (1);
        while (sp.size() < 3) sp.push_back (1.0);
        const size_t n = (size_t) dims[0] * dims[1] * dims[2];
        std::ifstream raw;
        std::ifstream* src = &h;
        if (datafile != "LOCAL")
        {
            std::string dir = name.substr (0, name.find_last_of ('/') + 1);
            raw.open (dir + datafile, std::ios::binary);
            if (!raw)
            {
                std::clog << "WARNING::interface: cannot open " << dir + datafile << std::endl;
                return false;
            }
            src = &raw;
        }
        else
        {
            h.seekg (data_pos);
        }
        std::vector<double> vals;
        if (type == "MET_UCHAR") read_raw<uint8_t> (*src, n, vals);
        else if (type == "MET_CHAR") read_raw<int8_t> (*src, n, vals);
        else if (type == "MET_USHORT") read_raw<uint16_t> (*src, n, vals);
        else if (type == "MET_SHORT") read_raw<int16_t> (*src, n, vals);
        else if (type == "MET_UINT") read_raw<uint32_t> (*src, n, vals);
        else if (type == "MET_INT") read_raw<int32_t> (*src, n, vals);
        else if (type == "MET_FLOAT") read_raw<float> (*src, n, vals);
        else if (type == "MET_DOUBLE") read_raw<double> (*src, n, vals);
        else
        {
            std::clog << "WARNING::interface: unsupported ElementType " << type << std::endl;
            return false;
        }
        // fastest axis first in the file: dims[0] = dimz, dims[2] = dimx
        stored.setdim ( (uint) dims[2], (uint) dims[1], (uint) dims[0]);
        stored.seth (sp[2], sp[1], sp[0]);
        for (size_t q = 0; q < n; ++q) stored.data() [q] = static_cast<S> (vals[q]);
        return true;
    }

    void convertfromimage3d (image3d<S> const& myim) { this->stored = myim; }
    void convert2image3d (image3d<S>& myim) const { myim = this->stored; }

    // graphics members: no graphics stack on this backend
    void setcolour (double const& = 1., double const& = 1., double const& = 0.) {}
    void setopacity (double const& = 0.5) {}
    void show_contour (double const& = 0) { headless ("show_contour"); }
    void show_image () { headless ("show_image"); }
    void show_image_and_contour (double const& = 0) { headless ("show_image_and_contour"); }
    void show_contour_with_background_image (interface&, double const& = 0)
    {
        headless ("show_contour_with_background_image");
    }
    void get_coordinates (uint& i, uint& j, uint& k) { (void) i; (void) j; (void) k; headless ("get_coordinates"); }
    void get_coordinates (uint& i1, uint& j1, uint& k1, uint& i2, uint& j2, uint& k2)
    {
        (void) i1; (void) j1; (void) k1; (void) i2; (void) j2; (void) k2;
        headless ("get_coordinates");
    }

    /* MetaImage writer: <imagename>.mhd + <imagename>.raw, MET_DOUBLE (the reference
     * also writes .jpg slices for 2-D images; only mhd is written here). */
    void write (std::string const& imagename = "image3d", std::string const& extension = "mhd") const
    {
        (void) extension;
        std::string base = imagename, rawname = imagename + ".raw";
        std::string rawfile = rawname.substr (rawname.find_last_of ('/') + 1);
        FILE* h = std::fopen ( (base + ".mhd").c_str(), "w");
        if (!h) return;
        std::fprintf (h, "ObjectType = Image\nNDims = 3\nBinaryData = True\n"
                      "BinaryDataByteOrderMSB = False\nDimSize = %u %u %u\n"
                      "ElementSpacing = %.17g %.17g %.17g\nElementType = MET_DOUBLE\n"
                      "ElementDataFile = %s\n", stored.getdimz(), stored.getdimy(), stored.getdimx(),
                      stored.gethz(), stored.gethy(), stored.gethx(), rawfile.c_str() );
        std::fclose (h);
        FILE* r = std::fopen (rawname.c_str(), "wb");
        if (!r) return;
        std::vector<double> buf (stored.size() );
        for (size_t q = 0; q < buf.size(); ++q) buf[q] = static_cast<double> (stored.data() [q]);
        std::fwrite (buf.data(), sizeof (double), buf.size(), r);
        std::fclose (r);
    }

private:
    static void headless (char const* what)
    {
        std::clog << "interface::" << what << ": unavailable (no graphics stack)" << std::endl;
    }
};

} // namespace im3d

#endif
