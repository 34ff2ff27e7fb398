/*
 * segmentation.hxx -- segm::segmentation<T>, the abstract base of the reference's
 * header/segmentation.hxx:50-165: the level `alpha`, the level-set function `phi`,
 * the headless interfaces `image` and `levelset`, apply() and getoutput().
 */
#ifndef IM3D_SEGMENTATION_HXX
#define IM3D_SEGMENTATION_HXX

#include "image3d.hxx"
#include "interface.hxx"

namespace segm
{

template <typename T>
class segmentation
{
protected:
    T alpha;
    im3d::interface<T> image;
    im3d::interface<T> levelset;
    im3d::image3d<T> phi;

public:
    segmentation () : alpha (0) {}
    virtual ~segmentation () {}

    virtual inline void set_alpha (T const& a) { this->alpha = a; }

    virtual void apply (im3d::image3d<T> const& myim, im3d::image3d<T> const& init) = 0;
    virtual void apply (im3d::image3d<T> const& myim) = 0;

    inline im3d::image3d<T> getoutput () const { return this->phi; }

    virtual inline void show_contour ()
    {
        levelset.convertfromimage3d (this->phi);
        levelset.show_contour (this->alpha);
    }
    virtual inline void show_levelset ()
    {
        levelset.convertfromimage3d (this->phi);
        levelset.show_image();
    }
    virtual inline void show_levelset_and_contour ()
    {
        levelset.convertfromimage3d (this->phi);
        levelset.show_image_and_contour (this->alpha);
    }
    virtual inline void show_levelset_with_background_image ()
    {
        levelset.convertfromimage3d (this->phi);
        levelset.show_contour_with_background_image (this->image, this->alpha);
    }
};

} // namespace segm

#endif
