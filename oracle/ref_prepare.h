// Scene preparation shared by the oracle's host and device drivers.
//
// TEST INFRASTRUCTURE ONLY (included by oracle/ref_harness.cpp and
// oracle/ref_gpu_harness.cu after the reference's Shading.cu and scene module
// headers).
#pragma once

namespace YMRT {

// SceneModule names GuiModule as a friend (src/core/SceneModule.h:87). The
// oracle is not linked with the GUI, so this class stands in for the part of
// GuiModule::UpdateScene that prepares a freshly parsed scene for rendering.
class GuiModule {
 public:
  static bool PrepareScene(SceneModule& m, const uint32_t* halton_perm, size_t perm_len, int width,
                           int height, std::vector<uint32_t>* instance_old_index) {
    std::unordered_map<uint32_t, uint32_t> dst_indices_map;
    TopBVHBuilder builder(m.primitive_instances.data(), (uint32_t)m.primitive_instances.size(),
                          m.transforms.data(), m.geometries.data());
    m.top_nodes.clear();
    builder.BuildSceneBVH(m.top_nodes, nullptr, nullptr, &dst_indices_map);
    for (auto& item : m.primitive_index_to_index_map) item.second = dst_indices_map[item.second];
    instance_old_index->assign(m.primitive_instances.size(), EMPTY_UINT32);
    for (auto& kv : dst_indices_map) (*instance_old_index)[kv.second] = kv.first;

    m.shape_lights.clear();
    m.shape_light_sample_table.clear();
    m.LoadShapeLight();

    m.permute_table.assign(halton_perm, halton_perm + perm_len);

    // the image tiles the host-side texture fetch reads (GuiModule::UpdateScene, src/core/GuiModule.cpp:237)
    m.image_tile_cache.image_tiles_host = m.image_texture_tiles.data();

    m.camera[EDITOR_CAMERA_INDEX].InitCameraRayTransfer(m.GetHostSceneDataPointer());
    std::memcpy(&m.camera[RENDERING_CAMERA_INDEX], &m.camera[EDITOR_CAMERA_INDEX], sizeof(Camera));
    m.camera[RENDERING_CAMERA_INDEX].m_width = width;
    m.camera[RENDERING_CAMERA_INDEX].m_height = height;
    m.camera[RENDERING_CAMERA_INDEX].SetAspectRatio(float(width) / float(height));
    return true;
  }
  // The part of GuiModule::UpdateScene a transform edit runs
  // (src/core/GuiModule.cpp:123-170): the top-level rebuild from the current
  // instance order, the light list, the camera's media stack.
  static void RebuildAfterTransformEdit(SceneModule& m, std::vector<uint32_t>* instance_old_index) {
    std::unordered_map<uint32_t, uint32_t> dst_indices_map;
    TopBVHBuilder builder(m.primitive_instances.data(), (uint32_t)m.primitive_instances.size(),
                          m.transforms.data(), m.geometries.data());
    m.top_nodes.clear();
    builder.BuildSceneBVH(m.top_nodes, nullptr, nullptr, &dst_indices_map);
    for (auto& item : m.primitive_index_to_index_map) item.second = dst_indices_map[item.second];
    std::vector<uint32_t> file_of(instance_old_index->size(), EMPTY_UINT32);
    for (auto& kv : dst_indices_map) file_of[kv.second] = (*instance_old_index)[kv.first];
    instance_old_index->swap(file_of);
    m.shape_lights.clear();
    m.shape_light_sample_table.clear();
    m.LoadShapeLight();
    m.camera[EDITOR_CAMERA_INDEX].InitCameraRayTransfer(m.GetHostSceneDataPointer());
    const int w = m.camera[RENDERING_CAMERA_INDEX].m_width, h = m.camera[RENDERING_CAMERA_INDEX].m_height;
    std::memcpy(&m.camera[RENDERING_CAMERA_INDEX], &m.camera[EDITOR_CAMERA_INDEX], sizeof(Camera));
    m.camera[RENDERING_CAMERA_INDEX].m_width = w;
    m.camera[RENDERING_CAMERA_INDEX].m_height = h;
    m.camera[RENDERING_CAMERA_INDEX].SetAspectRatio(float(w) / float(h));
  }
  static Scene HostScene(SceneModule& m) { return m.GetHostSceneDataPointer(); }
  static std::vector<GeometryData>& Geometries(SceneModule& m) { return m.geometries; }
  static std::vector<PrimitiveInstance>& Instances(SceneModule& m) { return m.primitive_instances; }
  static std::vector<ShapeLight>& Lights(SceneModule& m) { return m.shape_lights; }
  static std::vector<float>& LightTable(SceneModule& m) { return m.shape_light_sample_table; }
  static std::vector<glm::mat4>& Transforms(SceneModule& m) { return m.transforms; }
  static std::vector<glm::mat4>& InvTransforms(SceneModule& m) { return m.i_transforms; }
  static std::vector<TransformState>& TransformStates(SceneModule& m) { return m.transform_states; }
  static std::vector<Material>& Materials(SceneModule& m) { return m.materials; }
  static std::vector<Volume>& Volumes(SceneModule& m) { return m.volumes; }
  static std::vector<DistantLight>& DistantLights(SceneModule& m) { return m.distant_lights; }
  static std::vector<Texture>& Textures(SceneModule& m) { return m.textures; }
  static std::vector<ImageTile>& ImageTiles(SceneModule& m) { return m.image_texture_tiles; }
  static Camera* Cameras(SceneModule& m) { return m.camera; }
  static std::vector<TopNode>& TopNodes(SceneModule& m) { return m.top_nodes; }
};

}  // namespace YMRT
