// The drop-in example a caller of the reference's class writes against
// include/vmapping.h: construct, CreateMap, fuse from device and host
// buffers, render (library-allocated vertex map), mesh, surface points.
// Compiled (syntax only) by tests/test_headers.py.
#include "vmapping.h"  // -I include ; link -L voxelmapping_b200 -lvmap_b200 -lcudart

void drop_in_example(void* depth_dev, const unsigned char* rgb_host, const float* depth_host,
                     const vmap::Mat4f& cam_to_world)
{
    vmap::Mat3f K{{525, 0, 319.5f, 0, 525, 239.5f, 0, 0, 1}};
    vmap::VoxelMapping map(640, 480, K);  // VMAP_VOXEL_REF storage, colour on
    map.CreateMap(1 << 21, 1 << 20, 0.005f);
    map.FuseDepth(vmap::DeviceImage{depth_dev, 640 * 4, 480, 640}, cam_to_world);  // float metres; rows, cols
    map.FuseDepthAndImage(rgb_host, depth_host, cam_to_world);                     // host buffers
    vmap::DeviceImage vmap_img;  // empty: the library allocates it, as in the reference
    map.RenderScene(vmap_img, cam_to_world);
    float *verts, *norms;
    int n = map.Polygonize(verts, norms);  // library-owned host buffers, valid until the next call
    auto points = map.GetSurfacePoints();
    (void)n;
    (void)points;
}
