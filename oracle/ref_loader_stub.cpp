// Test infrastructure only: stand-ins for the reference's image loader
// (WindowsApp.Core ImageLoader, which needs LibRaw and stb_image, not built
// here), linked into oracle/_ref/libi360ref.so so that the reference's
// OverlapCulling.cpp links.  Every call reports that the file cannot be
// opened, which is the path the reference's own culling test exercises
// (WindowsApp.Tests/OverlapCullingTests.cpp:88-114: unknown dimensions ->
// the image is conservatively included).  No arithmetic of the reference is
// replaced.

#include "HeaderFiles/ImageLoader.h"

namespace WindowsApp::Core
{
struct ImageLoader::Impl
{
};

ImageLoader::ImageLoader() = default;
ImageLoader::~ImageLoader() = default;

bool ImageLoader::Open(const std::wstring&) { return false; }

bool ImageLoader::GetMetadata(ImageMetadata&) const { return false; }

bool GetStandardImageDimensions(const std::wstring&, int& outWidth, int& outHeight)
{
    outWidth = 0;
    outHeight = 0;
    return false;
}
}  // namespace WindowsApp::Core
