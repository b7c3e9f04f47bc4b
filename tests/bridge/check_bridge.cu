// Compiles the bridge of INTEGRATION.md section 2 (extracted into
// b200_bridge.cpp by tests/test_bridge_compile.py) against the reference's
// own CudaPayload / CudaHosekSky / CudaCamera / CudaSpec and checks, on the
// host, that each mirror carries every field of Noor's objects into the
// library's structs, then that the bridge resolves all of the library's
// entry points from libnoor_b200.so.  Prints "bridge ok" on success.
#include "b200_bridge.cpp"

#include <cmath>

static int failures = 0;
#define EXPECT(c)                                                            \
    do {                                                                     \
        if (!(c)) {                                                          \
            std::fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
            ++failures;                                                      \
        }                                                                    \
    } while (0)

static bool eq3(const float* a, const float3& b) { return a[0] == b.x && a[1] == b.y && a[2] == b.z; }

int main() {
    using namespace b200;
    using nb::NOOR_CAMERA_PERSP;
    using nb::NOOR_SKY_PHYSICAL;
    using nb::NOOR_ISECT_REF_WALD;
    using nb::NOOR_FILM_REF_LERP;
    using nb::NOOR_FILTER_POINT;
    using nb::NOOR_FILTER_LINEAR;
    using nb::NOOR_ADDRESS_CLAMP;
    // ---- payload: two triangles, two instances, three nodes, textures of
    // 4, 3 and 1 channels, two materials and one light of each kind
    auto P = std::make_unique<CudaPayload>();
    P->_num_triangles = 2;
    P->_attribute_indices = {glm::uvec4(0, 1, 2, 0), glm::uvec4(2, 1, 3, 1)};
    for (int i = 0; i < 4; ++i) {
        P->_vertices.push_back(glm::vec4(i, 2.0f * i, -1.0f * i, 1.0f));
        P->_normals.push_back(glm::vec4(0.0f, 1.0f, 0.5f * i, 0.0f));
        P->_uvs.push_back(glm::vec2{0.25f * i, 1.0f - 0.25f * i});
    }
    std::vector<glm::vec4>* rows[9] = {&P->_normal_row0,          &P->_normal_row1,          &P->_normal_row2,
                                       &P->_world_to_object_row0, &P->_world_to_object_row1, &P->_world_to_object_row2,
                                       &P->_object_to_world_row0, &P->_object_to_world_row1, &P->_object_to_world_row2};
    for (int k = 0; k < 9; ++k)
        for (int i = 0; i < 2; ++i) rows[k]->push_back(glm::vec4(k, i, k * i, 1.0f + k));
    for (int i = 0; i < 2; ++i) {
        P->_wald_ax_nu_nv_nd.push_back(glm::uvec4(10 + i, 11, 12, 13));
        P->_wald_bnu_bnv_au_av.push_back(glm::uvec4(20 + i, 21, 22, 23));
        P->_wald_cnu_cnv_deg_mat.push_back(glm::uvec4(30 + i, 31, 32, 33));
    }
    P->_bvh_root_node = 2;
    for (int i = 0; i < 3; ++i) {
        P->_bvh_min_right_start_nodes.push_back(glm::uvec4(100 + i, 101, 102, 103));
        P->_bvh_max_axis_count_nodes.push_back(glm::uvec4(200 + i, 201, 202, 203));
    }
    P->_textures.emplace_back(make_float3(0.5f, 0.25f, 0.125f));   // a constant colour (3 -> 4 channels)
    P->_textures.emplace_back(0.75f);                               // the metalness float (1 channel)
    P->_textures.emplace_back(4, 2, 4, cudaFilterModeLinear, cudaAddressModeClamp);   // an env map
    float* env = const_cast<float*>(P->_textures.back().getData());
    for (int i = 0; i < 32; ++i) env[i] = 0.5f * i;
    for (int i = 0; i < 2; ++i) {
        CudaMaterial c;
        c._diffuse_uvscale = make_float2(1.0f + i, 2.0f);
        c._metalness_uvscale = make_float2(3.0f, 4.0f + i);
        c._diffuse_tex_idx = 1 + i;
        c._metalness_tex_idx = 1;
        c._transparency_tex_idx = 0;
        c._bumpfactor = 0.5f;
        c._emitter_scale = 3.0f + i;
        c._coat_roughness = 0.01f;
        c._coat_ior = 1.4f;
        c._type = i ? METAL : DIFFUSE;
        P->_materials.push_back(c);
    }
    CudaShape s;
    s._center = make_float3(1, 2, 3);
    s._u = make_float3(1, 0, 0);
    s._v = make_float3(0, 0, 1);
    s._n = make_float3(0, -1, 0);
    s._area = 1.0f;
    s._radius = 0.5f;
    s._radius2 = 0.25f;
    s._light_idx = 0;
    s._type = QUAD;
    P->_area_light_data.emplace_back(s, make_float3(5, 6, 7), true);
    P->_num_area_lights = 1;
    P->_point_light_data.emplace_back(make_float3(1, 1, 1), make_float3(2, 3, 4));
    P->_num_point_lights = 1;
    P->_spot_light_data.emplace_back(make_float3(0, 3, 0), make_float3(0, -1, 0), make_float3(9, 9, 9), 0.9f, 0.8f);
    P->_num_spot_lights = 1;
    P->_distant_light_data.emplace_back(make_float3(0, 3, 4), make_float3(1, 1, 0.5f));
    P->_num_distant_lights = 1;
    P->_infinite_light_data.emplace_back(1.0f);
    P->_num_infinite_lights = 1;

    mirror_payload(*P);
    const noor_payload& g = m.payload;
    EXPECT(g.num_triangles == 2 && g.num_vertices == 4 && g.num_instances == 2 && g.num_bvh_nodes == 3);
    EXPECT(g.attribute_indices[4] == 2 && g.attribute_indices[7] == 1);
    EXPECT(g.vertices[4 * 3 + 1] == 6.0f && g.normals[4 * 2 + 2] == 1.0f && g.uvs[2 * 3 + 1] == 0.25f);
    for (int k = 0; k < 9; ++k) {
        const float* r = k < 3 ? g.normal_row[k] : (k < 6 ? g.world_to_object_row[k - 3] : g.object_to_world_row[k - 6]);
        EXPECT(r[4 + 0] == (float)k && r[4 + 1] == 1.0f && r[4 + 2] == (float)k && r[4 + 3] == 1.0f + k);
    }
    EXPECT(g.wald_ax_nu_nv_nd[4] == 11 && g.wald_bnu_bnv_au_av[5] == 21 && g.wald_cnu_cnv_deg_mat[7] == 33);
    EXPECT(g.bvh_root_node == 2 && g.bvh_min_right_start[8] == 102 && g.bvh_max_axis_count[11] == 203);
    EXPECT(g.num_textures == 3);
    EXPECT(g.textures[0].width == 1 && g.textures[0].rgba[0] == 0.5f && g.textures[0].rgba[2] == 0.125f);
    EXPECT(g.textures[1].rgba[0] == 0.75f && g.textures[1].rgba[1] == 0.0f && g.textures[1].rgba[3] == 1.0f);
    EXPECT(g.textures[2].width == 4 && g.textures[2].height == 2 && g.textures[2].rgba[31] == 15.5f);
    EXPECT(g.textures[0].filter == NOOR_FILTER_POINT && g.textures[0].address == NOOR_ADDRESS_CLAMP);
    EXPECT(g.textures[2].filter == NOOR_FILTER_LINEAR && g.textures[2].address == NOOR_ADDRESS_CLAMP);
    EXPECT(g.num_materials == 2);
    const noor_material& mt = g.materials[1];
    EXPECT(mt.diffuse_uvscale[0] == 2.0f && mt.metalness_uvscale[1] == 5.0f && mt.diffuse_tex_idx == 2);
    EXPECT(mt.metalness_tex_idx == 1 && mt.bumpfactor == 0.5f && mt.emitter_scale == 4.0f);
    EXPECT(mt.coat_roughness == 0.01f && mt.coat_ior == 1.4f && mt.coat_weight == 1.0f && mt.type == METAL);
    EXPECT(g.num_area_lights == 1 && eq3(g.area_lights[0].shape.center, s._center) &&
           eq3(g.area_lights[0].shape.n, s._n) && g.area_lights[0].shape.radius2 == 0.25f &&
           g.area_lights[0].two_sided == 1 && g.area_lights[0].ke[2] == 7.0f);
    EXPECT(g.num_point_lights == 1 && g.point_lights[0].ke[1] == 3.0f && g.point_lights[0].position[0] == 1.0f);
    EXPECT(g.num_spot_lights == 1 && g.spot_lights[0].direction[1] == -1.0f && g.spot_lights[0].cos_inner == 0.9f &&
           g.spot_lights[0].cos_outer == 0.8f && g.spot_lights[0].ke[0] == 9.0f);
    EXPECT(g.num_distant_lights == 1 && std::fabs(g.distant_lights[0].direction[1] - 0.6f) < 1e-6f &&
           g.distant_lights[0].ke[2] == 0.5f);
    EXPECT(g.num_infinite_lights == 1);

    // ---- sky
    CudaHosekSky H;
    std::memset(&H, 0, sizeof(H));
    CudaArHosekSkyModelState* st[3] = {&H._state_r, &H._state_g, &H._state_b};
    for (int c = 0; c < 3; ++c) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 9; ++j) st[c]->_configs[i][j] = 100.0f * c + 10.0f * i + j;
        st[c]->_radiances.x = 1.0f + c;
        st[c]->_turbidity = 3.0f;
        st[c]->_solar_radius = 0.0045f;
        st[c]->_emission_correction_factor_sun.z = 2.0f + c;
        st[c]->_albedo = 0.3f;
        st[c]->_elevation = 0.5f + c;
    }
    H._solar_dir = make_float3(0, 0.5f, 0.866f);
    H._ground_albedo = make_float3(0.3f, 0.3f, 0.3f);
    H._solar_scale = 250.0f;
    H._solar_radius = 0.009f;
    mirror_sky(H);
    EXPECT(m.sky.state[2].configs[1][4] == 214.0f && m.sky.state[1].radiances[0] == 2.0f);
    EXPECT(m.sky.state[0].turbidity == 3.0f && m.sky.state[2].emission_correction_factor_sun[2] == 4.0f);
    EXPECT(m.sky.state[1].elevation == 1.5f && m.sky.state[2].albedo == 0.3f);
    EXPECT(eq3(m.sky.solar_dir, H._solar_dir) && m.sky.solar_scale == 250.0f && m.sky.solar_radius == 0.009f);

    // ---- camera: transforms read back through CudaTransform's interface
    CudaCamera C;
    C._cameraToWorld = CudaTransform(make_float4(1, 2, 3, 4), make_float4(5, 6, 7, 8), make_float4(9, 10, 11, 12));
    C._rasterToCamera = CudaTransform(make_float4(0.5f, 0, 0, -1), make_float4(0, -0.5f, 0, 1),
                                      make_float4(0, 0, 0, -1));
    C._worldToRaster = CudaTransform(make_float4(2, 0, 0, 0), make_float4(0, 2, 0, 0), make_float4(0, 0, 2, 0));
    C._dxCamera = make_float3(0.5f, 0, 0);
    C._dyCamera = make_float3(0, -0.5f, 0);
    C._lens_radius = 0.0f;
    C._focal_length = 3.75f;
    C._image_area = 4.0f;
    C._w = 640;
    C._h = 480;
    C._center = 640 * 240 + 320;
    C._type = PERSP;
    mirror_camera(C);
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 4; ++k) EXPECT(m.camera.camera_to_world[r][k] == 4.0f * r + k + 1);
    EXPECT(m.camera.raster_to_camera[1][1] == -0.5f && m.camera.raster_to_camera[0][3] == -1.0f &&
           m.camera.raster_to_camera[2][3] == -1.0f && m.camera.world_to_raster[2][2] == 2.0f);
    EXPECT(m.camera.dy_camera[1] == -0.5f && m.camera.focal_length == 3.75f && m.camera.image_area == 4.0f);
    EXPECT(m.camera.w == 640 && m.camera.h == 480 && m.camera.center == C._center &&
           m.camera.type == NOOR_CAMERA_PERSP);

    // ---- spec
    CudaSpec S;
    std::memset(&S, 0, sizeof(S));
    S._reflection_bias = 1e-4f;
    S._shadow_bias = 2e-4f;
    S._world_radius = 10.0f;
    S._wr2 = 100.0f;
    S._bvh_root_node = 2;
    S._lighting_type = 7;
    S._bounces = 5;
    S._rr = 3;
    S._bvh_height = 17;
    S._num_gpus = 1;
    S._skydome_type = PHYSICAL;
    S._mis = true;
    mirror_spec(S);
    EXPECT(m.spec.reflection_bias == 1e-4f && m.spec.shadow_bias == 2e-4f && m.spec.wr2 == 100.0f);
    EXPECT(m.spec.bvh_root_node == 2 && m.spec.lighting_type == 7 && m.spec.bounces == 5 && m.spec.rr == 3);
    EXPECT(m.spec.bvh_height == 17 && m.spec.num_gpus == 1 && m.spec.skydome_type == NOOR_SKY_PHYSICAL);
    EXPECT(m.spec.mis == 1 && m.spec.debug_sky == 0 && m.spec.intersector == NOOR_ISECT_REF_WALD &&
           m.spec.film_mode == NOOR_FILM_REF_LERP);

    // ---- the library's entry points resolve (no call is made: no GPU here)
    const Api& a = api();
    EXPECT(a.load_cuda_data && a.update_cuda_camera && a.update_cuda_hosek && a.update_cuda_spec &&
           a.cuda_path_tracer && a.debug_skydome && a.device_free_memory && a.get_lookAt && a.get_framebuffer &&
           a.last_error);
    if (failures) return 1;
    std::printf("bridge ok\n");
    return 0;
}
