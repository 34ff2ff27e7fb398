// rsfe_splitbregman -- command-line segmentation on the B200 backend, with the
// arguments and flow of the reference's examples/rsfe_splitbregman.cxx:34-117:
//
//   rsfe_splitbregman <image.mhd> [<getpotfile> [<logfilename> [<init.mhd>]]]
//
// reads the volume, rescales it to [0, 255], loads the parameters of section
// splitbregman/init/ of the GetPot file (default ./data) and runs apply (from the
// default cube, or from the initial level set given as fourth argument). The level set
// is written as <outputname>_<iterations>_final.mhd when dumpfrequency > 0, as in the
// reference; display (showfrequency) is not available without a graphics stack.
#include <iostream>
#include <string>

#include "im3d/image3d.hxx"
#include "im3d/interface.hxx"
#include "im3d/rsfe_splitbregman.hxx"

typedef double MY_REAL;

int main (int argc, char** argv)
{
    std::string filename, getpotfile = "./data", logfilename = "!", initname = "!";
    if (argc < 2)
    {
        std::cout << "\n\t*** rsfe_splitbregman helper ***\n\n"
                  << "\trsfe_splitbregman <name of image to segment>\n"
                  << "\t\t\t[<getpotfile> <logfilename> <init phi filename>]\n\n"
                  << "\t<getpotfile> is the \".pot\" to import parameters of algorithm.\n"
                  << "\tDefault value is \"./data\".\n\n"
                  << "\t<logfilename> is name of logfile where history is saved.\n"
                  << "\tIf it is not set terminal is used.\n\n"
                  << "\t<init phi filename> is name of image with whom you'd like to initialize phi.\n"
                  << "\tIf it is not set default cube is used.\n" << std::endl;
        return 0;
    }
    filename = argv[1];
    if (argc > 2) getpotfile = argv[2];
    if (argc > 3) logfilename = argv[3];
    if (argc > 4) initname = argv[4];
    std::cout << "you have selected: " << filename << std::endl;

    im3d::image3d<MY_REAL> myim, init;
    {
        im3d::interface<MY_REAL> reader;
        if (!reader.load (filename) ) return 1;
        reader.convert2image3d (myim);
    }
    myim.change_range_of_intensity (255);
    if (initname != "!")
    {
        im3d::interface<MY_REAL> reader;
        if (!reader.load (initname) ) return 1;
        reader.convert2image3d (init);
    }

    segm::rsfe_splitbregman<MY_REAL> algo;
    algo.set_getpotfile (getpotfile);
    algo.set_onthego (true);
    if (logfilename != "!") algo.set_logfilename (logfilename);
    std::cout << "Applying segmentation algorithm ..." << std::endl;
    if (initname == "!") algo.apply (myim);
    else algo.apply (myim, init);
    const im3d_rsfe_stats& st = algo.get_stats();
    std::cout << "iterations " << st.iterations << " last_tol " << st.last_tol << " sweeps "
              << st.total_sweeps << std::endl;
    return 0;
}
