// scene_pack.cu -- host-side packing of a vt_scene_desc into the device
// layouts (scenePack.ts packSceneFromCore:1104-1310 restated for the wide
// BVH): per-triangle records and 8-wide nodes (one tree, or per-mesh bottom
// levels under a top level over the instances), materials, the area-light
// CDF, point lights and the environment with its importance CDFs.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "scene_pack.h"
#include "light_tree.h"
#include "pt_kernels.h"

namespace vt {

namespace {
double luminance(const float* c) { return 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]; }
}  // namespace

bool invert4(const double* m, double* inv) {  // any layout, Gauss-Jordan with partial pivoting
  double a[4][8];
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      a[r][c] = m[r * 4 + c];
      a[r][c + 4] = r == c ? 1.0 : 0.0;
    }
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
    if (!(std::fabs(a[piv][c]) > 1e-300)) return false;
    if (piv != c)
      for (int k = 0; k < 8; ++k) std::swap(a[c][k], a[piv][k]);
    const double d = a[c][c];
    for (int k = 0; k < 8; ++k) a[c][k] /= d;
    for (int r = 0; r < 4; ++r) {
      if (r == c) continue;
      const double f = a[r][c];
      for (int k = 0; k < 8; ++k) a[r][k] -= f * a[c][k];
    }
  }
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) inv[r * 4 + c] = a[r][c + 4];
  return true;
}

namespace {
void mat_mul_cm(const double* a, const double* b, double* out) {  // column-major 4x4: out = a * b
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += a[k * 4 + r] * b[c * 4 + k];
      out[c * 4 + r] = s;
    }
}


}  // namespace

// inverse(P * V) as a row-major float matrix
void inverse_view_proj(const float* view, const float* proj, float* out_rm) {
  double v[16], p[16], vp[16], rm[16], inv[16];
  for (int i = 0; i < 16; ++i) { v[i] = view[i]; p[i] = proj[i]; }
  mat_mul_cm(p, v, vp);
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) rm[r * 4 + c] = vp[c * 4 + r];
  if (!invert4(rm, inv)) fail(VT_ERR_INVALID_ARGUMENT, "camera view-projection matrix is singular");
  for (int i = 0; i < 16; ++i) out_rm[i] = (float)inv[i];
}

void view_proj(const float* view, const float* proj, float* out_rm) {
  double v[16], p[16], vp[16];
  for (int i = 0; i < 16; ++i) { v[i] = view[i]; p[i] = proj[i]; }
  mat_mul_cm(p, v, vp);
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) out_rm[r * 4 + c] = (float)vp[c * 4 + r];
}



InstanceSet place_instances(const vt_instance_desc* insts, size_t ni, const std::vector<pt::Material>& mats,
                            const std::vector<uint32_t>& blas_root,
                            const std::vector<std::array<double, 6>>& local_box) {
  // world-to-local rows and world AABBs (transformAabb, scenePack.ts:197-223)
  InstanceSet out;
  out.recs.resize(ni);
  out.aabbs.resize(6 * ni);
  out.rows.reserve(12 * ni);
  for (size_t i = 0; i < ni; ++i) {
    const vt_instance_desc& id = insts[i];
    if (id.mesh >= blas_root.size())
      fail(VT_ERR_RANGE, "instance " + std::to_string(i) + " references mesh " + std::to_string(id.mesh));
    if (id.material >= mats.size())
      fail(VT_ERR_RANGE, "instance " + std::to_string(i) + " references material " + std::to_string(id.material));
    if (mats[id.material].emissive) fail(VT_ERR_INVALID_ARGUMENT, "emissive materials are not supported on instances");
    double rm[16], inv[16];
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) rm[r * 4 + c] = id.local_to_world[c * 4 + r];
    for (double x : rm)
      if (!std::isfinite(x)) fail(VT_ERR_RANGE, "instance " + std::to_string(i) + " transform is not finite");
    if (!invert4(rm, inv)) fail(VT_ERR_INVALID_ARGUMENT, "instance " + std::to_string(i) + " is not invertible");
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) out.rows.push_back(id.local_to_world[c * 4 + r]);
    InstanceRecord& rec = out.recs[i];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) rec.w2l[4 * r + c] = (float)inv[r * 4 + c];
    rec.blas_root = blas_root[id.mesh];
    rec.instance_id = (uint32_t)i;
    rec.material = id.material;
    rec.pad = mats[id.material].flags;
    const auto& lb = local_box[id.mesh];
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < 8; ++c) {
      const double q[3] = {(c & 1) ? lb[3] : lb[0], (c & 2) ? lb[4] : lb[1], (c & 4) ? lb[5] : lb[2]};
      for (int k = 0; k < 3; ++k) {
        const double v = rm[k * 4] * q[0] + rm[k * 4 + 1] * q[1] + rm[k * 4 + 2] * q[2] + rm[k * 4 + 3];
        mn[k] = std::min(mn[k], v);
        mx[k] = std::max(mx[k], v);
      }
    }
    for (int k = 0; k < 3; ++k) { out.aabbs[6 * i + k] = mn[k]; out.aabbs[6 * i + 3 + k] = mx[k]; }
  }
  return out;
}

void refit_tlas_host(BinaryBvhHost& tl, const double* aabbs, size_t n) {
  // refitTlas (shared-bvh/src/tlas.ts:990-1012): same topology and leaf
  // assignment; leaves take the union of their instances' AABBs (stored as f32
  // like a build), interior nodes the union of their children, bottom-up
  // (preorder: children come after their parent)
  for (size_t i = tl.nodes.size(); i-- > 0;) {
    BinaryNode& nd = tl.nodes[i];
    if (is_leaf_word(nd.w7)) {
      double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
      const uint32_t first = nd.w6, count = nd.w7 & 0xFFFFu;
      for (uint32_t j = 0; j < count; ++j) {
        const uint32_t inst = tl.reordered_to_source[first + j];
        if (inst >= n) fail(VT_ERR_BUILD, "top-level leaf references instance " + std::to_string(inst));
        for (int k = 0; k < 3; ++k) {
          mn[k] = std::min(mn[k], aabbs[6 * inst + k]);
          mx[k] = std::max(mx[k], aabbs[6 * inst + 3 + k]);
        }
      }
      for (int k = 0; k < 3; ++k) {
        nd.mn[k] = (float)mn[k];
        nd.mx[k] = (float)mx[k];
      }
    } else {
      const BinaryNode &l = tl.nodes[i + 1], &r = tl.nodes[i + nd.w6];
      for (int k = 0; k < 3; ++k) {
        nd.mn[k] = std::min(l.mn[k], r.mn[k]);
        nd.mx[k] = std::max(l.mx[k], r.mx[k]);
      }
    }
  }
}

void append_mesh(const vt_mesh_desc& md, size_t m, size_t material_count, std::vector<float>& pos,
                 std::vector<uint32_t>& idx, std::vector<uint32_t>& tri_mat) {
  if (md.material >= material_count)
    fail(VT_ERR_RANGE, "mesh " + std::to_string(m) + " references material " + std::to_string(md.material));
  if ((md.vertex_count && !md.positions) || (md.triangle_count && !md.indices))
    fail(VT_ERR_INVALID_ARGUMENT, "mesh " + std::to_string(m) + " has null arrays");
  const uint32_t base = (uint32_t)(pos.size() / 4);
  for (size_t v = 0; v < md.vertex_count; ++v) {
    for (int k = 0; k < 3; ++k) {
      const float x = md.positions[3 * v + k];
      if (!std::isfinite(x)) fail(VT_ERR_RANGE, "mesh " + std::to_string(m) + " has a non-finite position");
      pos.push_back(x);
    }
    pos.push_back(0.0f);
  }
  for (size_t t = 0; t < md.triangle_count; ++t) {
    for (int k = 0; k < 3; ++k) {
      const uint32_t i = md.indices[3 * t + k];
      if (i >= md.vertex_count) fail(VT_ERR_RANGE, "mesh " + std::to_string(m) + " index out of range");
      idx.push_back(base + i);
    }
    idx.push_back(0u);
    tri_mat.push_back(md.material);
  }
}

// The engine's tree over vertices pos (4 floats each) and triangles idx (4
// u32 each): the binned-SAH build and the SAH-optimal 8-wide encoding, on the
// GPU or on the host (the same words either way).
static void build_tree(const SceneBuild& sb, const std::vector<float>& pos, const std::vector<uint32_t>& idx,
                       const uint32_t* tri_mat, uint32_t node_base, uint32_t rec_base, int max_leaf,
                       BinaryBvhHost& bin, WideBvhHost& wide) {
  BuildOptions bo;
  bo.max_leaf = max_leaf;
  bo.bins = kEngineBins;
  WideCollapse collapse = kEngineCollapse;
  collapse.width = sb.bvh_width;
  const size_t ntri = idx.size() / 4;
  if (sb.gpu) {
    DeviceScope ds(sb.device);
    ScratchBuffer<float> dpos(std::max<size_t>(pos.size(), 1), sb.stream);
    ScratchBuffer<uint32_t> didx(std::max<size_t>(idx.size(), 1), sb.stream), dmat(std::max<size_t>(ntri, 1), sb.stream);
    if (!pos.empty()) VT_CUDA(cudaMemcpyAsync(dpos.ptr, pos.data(), pos.size() * 4, cudaMemcpyHostToDevice, sb.stream));
    if (!idx.empty()) VT_CUDA(cudaMemcpyAsync(didx.ptr, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice, sb.stream));
    if (ntri && tri_mat) VT_CUDA(cudaMemcpyAsync(dmat.ptr, tri_mat, ntri * 4, cudaMemcpyHostToDevice, sb.stream));
    BinaryBvhDevice bd;
    bin = build_binary_gpu(dpos.ptr, pos.size(), didx.ptr, idx.size(), bo, sb.stream, &bd);
    wide = encode_wide_gpu(bd, dpos.ptr, 4, didx.ptr, 4, tri_mat ? dmat.ptr : nullptr, node_base, rec_base,
                           &collapse, nullptr, sb.stream);
  } else {
    bin = build_binary_host(pos.data(), pos.size(), idx.data(), idx.size(), bo);
    wide = encode_wide(bin, pos.data(), 4, idx.data(), 4, tri_mat, node_base, rec_base, &collapse);
  }
  if (sb.validate) {
    validate_binary(bin, (int64_t)ntri);
    validate_wide(wide.nodes.data(), wide.nodes.size() / 20, wide.tris.data(), wide.tris.size() / 16, node_base, ntri,
                  false, kTraversalStack, node_base, rec_base);
  }
}

BinaryBvhHost build_top_level(const SceneBuild& sb, const double* aabbs, size_t n) {
  if (!sb.gpu) return build_tlas_host(aabbs, n);
  DeviceScope ds(sb.device);
  return build_tlas_gpu(aabbs, n, 1, 16, kMaxBinaryDepth, sb.stream);
}

WideBvhHost encode_top_level(const SceneBuild& sb, const BinaryBvhHost& tl, const std::vector<InstanceRecord>& recs,
                             uint32_t root) {
  if (!sb.gpu) return encode_wide_tlas(tl, recs.data(), root);
  DeviceScope ds(sb.device);
  BinaryBvhDevice bd;
  bd.n_nodes = tl.nodes.size();
  bd.ntri = tl.reordered_to_source.size();
  bd.nodes.resize(std::max<size_t>(bd.n_nodes, 1));
  bd.order.resize(std::max<size_t>(bd.ntri, 1));
  ScratchBuffer<float> drecs(std::max<size_t>(16 * recs.size(), 1), sb.stream);
  if (bd.n_nodes)
    VT_CUDA(cudaMemcpyAsync(bd.nodes.ptr, tl.nodes.data(), bd.n_nodes * sizeof(BinaryNode), cudaMemcpyHostToDevice,
                            sb.stream));
  if (bd.ntri)
    VT_CUDA(cudaMemcpyAsync(bd.order.ptr, tl.reordered_to_source.data(), bd.ntri * 4, cudaMemcpyHostToDevice,
                            sb.stream));
  if (!recs.empty())
    VT_CUDA(cudaMemcpyAsync(drecs.ptr, recs.data(), recs.size() * sizeof(InstanceRecord), cudaMemcpyHostToDevice,
                            sb.stream));
  return encode_wide_gpu(bd, nullptr, 4, nullptr, 4, nullptr, root, 0, nullptr, drecs.ptr, sb.stream);
}

BlasPack pack_blas(const std::vector<float>& pos, const std::vector<uint32_t>& idx, uint32_t material,
                   uint32_t node_base, uint32_t rec_base, int max_leaf, const SceneBuild& sb) {
  const size_t ntri = idx.size() / 4;
  std::vector<uint32_t> mm(ntri, material);
  BinaryBvhHost b;
  BlasPack out;
  build_tree(sb, pos, idx, mm.data(), node_base, rec_base, max_leaf, b, out.wide);
  const BinaryNode& rn = b.nodes[0];
  out.local_box = {rn.mn[0], rn.mn[1], rn.mn[2], rn.mx[0], rn.mx[1], rn.mx[2]};
  if (ntri == 0) out.local_box = {0, 0, 0, 0, 0, 0};
  return out;
}

PackedScene pack_scene(const vt_scene_desc* sc, uint32_t node_base, uint32_t rec_base, int max_leaf,
                       const SceneBuild& sb) {
  if (!sc) fail(VT_ERR_INVALID_ARGUMENT, "scene is null");
  if (sc->mesh_count && !sc->meshes) fail(VT_ERR_INVALID_ARGUMENT, "meshes is null");
  if (sc->material_count && !sc->materials) fail(VT_ERR_INVALID_ARGUMENT, "materials is null");
  if (sc->point_light_count && !sc->point_lights) fail(VT_ERR_INVALID_ARGUMENT, "point_lights is null");
  PackedScene p;
  std::vector<float> pos;
  std::vector<uint32_t> idx, tri_mat;
  for (size_t m = 0; m < sc->mesh_count; ++m) append_mesh(sc->meshes[m], m, sc->material_count, pos, idx, tri_mat);
  // materials
  std::vector<pt::Material> mats(sc->material_count);
  for (size_t i = 0; i < sc->material_count; ++i) {
    const vt_material_desc& d = sc->materials[i];
    pt::Material& m = mats[i];
    m.base_color = make_float3(d.base_color[0], d.base_color[1], d.base_color[2]);
    m.roughness = d.roughness;
    m.emission = make_float3(d.emission[0], d.emission[1], d.emission[2]);
    auto unit = [&](float v, const char* what) {
      if (!(v >= 0.0f && v <= 1.0f))
        fail(VT_ERR_RANGE, "material " + std::to_string(i) + ": " + what + " must be in [0, 1]");
      return v;
    };
    unit(d.roughness, "roughness");
    m.metallic = unit(d.metallic, "metallic");
    m.transmission = unit(d.transmission, "transmission");
    m.specular = unit(d.specular_intensity, "specular_intensity");
    if (!(d.ior >= 0.0f) || !std::isfinite(d.ior)) fail(VT_ERR_RANGE, "material " + std::to_string(i) + ": ior must be >= 0");
    m.ior = d.ior > 0.0f ? std::max(d.ior, 1.0f) : 1.5f;  // materialPacking.ts:130-131 (0 here: the 1.5 default)
    const float ratio = (m.ior - 1.0f) / (m.ior + 1.0f);
    m.f0_ior = ratio * ratio * m.specular;
    m.kind = (d.transmission > 0.0f && d.metallic == 0.0f) ? pt::kDielectric
                                                           : (d.metallic > 0.0f ? pt::kMetal : pt::kOpaque);
    m.alpha = std::max(d.roughness * d.roughness, 1e-3f);
    m.emissive = (d.emission[0] > 0.0f || d.emission[1] > 0.0f || d.emission[2] > 0.0f) ? 1u : 0u;
    if (d.flags & ~3u) fail(VT_ERR_INVALID_ARGUMENT, "material " + std::to_string(i) + " has unknown flags");
    m.flags = d.flags;
  }
  const size_t ntri = tri_mat.size();
  // geometry
  const bool two_level = sc->instance_count > 0;
  if (two_level && !sc->instances) fail(VT_ERR_INVALID_ARGUMENT, "instances is null");
  std::vector<uint32_t> node_words;
  std::vector<float> rec_floats, inst_lanes, inst_tab, inst_rows;
  int depth = 1;
  uint32_t root = 0;
  if (!two_level) {
    WideBvhHost w;
    build_tree(sb, pos, idx, tri_mat.data(), node_base, rec_base, max_leaf, p.binary, w);
    node_words = std::move(w.nodes);
    rec_floats = std::move(w.tris);
    depth = w.depth;
    // material flags of each triangle record in its free word (v2.w); padding records stay 0
    for (size_t r = 0; r + 16 <= rec_floats.size(); r += 16) {
      if (rec_floats[r + 15] == 0.0f) continue;
      uint32_t mat;
      std::memcpy(&mat, &rec_floats[r + 7], 4);
      const uint32_t fl = mat < mats.size() ? mats[mat].flags : 0u;
      std::memcpy(&rec_floats[r + 11], &fl, 4);
    }
  } else {
    // one bottom-level tree per mesh, in the mesh's own space, concatenated
    std::vector<uint32_t> blas_root(sc->mesh_count), rec_start(sc->mesh_count);
    std::vector<std::array<double, 6>> local_box(sc->mesh_count);
    std::vector<int> depths(sc->mesh_count);
    int blas_depth = 1;
    size_t vbase = 0, tbase = 0;
    for (size_t m = 0; m < sc->mesh_count; ++m) {
      const vt_mesh_desc& md = sc->meshes[m];
      std::vector<float> mp(pos.begin() + 4 * vbase, pos.begin() + 4 * (vbase + md.vertex_count));
      std::vector<uint32_t> mi(idx.begin() + 4 * tbase, idx.begin() + 4 * (tbase + md.triangle_count));
      for (size_t t = 0; t < md.triangle_count; ++t)
        for (int k = 0; k < 3; ++k) mi[4 * t + k] -= (uint32_t)vbase;
      blas_root[m] = (uint32_t)(node_words.size() / 20);
      rec_start[m] = (uint32_t)(rec_floats.size() / 16);
      BlasPack bp = pack_blas(mp, mi, md.material, blas_root[m], rec_start[m], max_leaf, sb);
      node_words.insert(node_words.end(), bp.wide.nodes.begin(), bp.wide.nodes.end());
      rec_floats.insert(rec_floats.end(), bp.wide.tris.begin(), bp.wide.tris.end());
      depths[m] = bp.wide.depth;
      blas_depth = std::max(blas_depth, bp.wide.depth);
      local_box[m] = bp.local_box;
      vbase += md.vertex_count;
      tbase += md.triangle_count;
    }
    p.blas_rec_start = std::move(rec_start);
    p.blas_depths = std::move(depths);
    if (sc->instance_count && !sc->instances) fail(VT_ERR_INVALID_ARGUMENT, "instances is null");
    const size_t ni = sc->instance_count;
    InstanceSet placed = place_instances(sc->instances, ni, mats, blas_root, local_box);
    std::vector<InstanceRecord>& recs = placed.recs;
    std::vector<double>& aabbs = placed.aabbs;
    inst_rows = std::move(placed.rows);
    BinaryBvhHost tl = build_top_level(sb, aabbs.data(), ni);
    root = (uint32_t)(node_words.size() / 20);
    WideBvhHost tw = encode_top_level(sb, tl, recs, root);
    if (sb.validate) {
      validate_binary(tl, (int64_t)ni);
      validate_wide(tw.nodes.data(), tw.nodes.size() / 20, tw.tris.data(), tw.tris.size() / 16, root, ni, true,
                    kTraversalStack, root, 0);
    }
    node_words.insert(node_words.end(), tw.nodes.begin(), tw.nodes.end());
    inst_lanes = std::move(tw.tris);
    inst_tab.resize(16 * ni);
    std::memcpy(inst_tab.data(), recs.data(), ni * sizeof(InstanceRecord));
    depth = tw.depth + blas_depth;
    p.binary = std::move(tl);
    p.blas_root = std::move(blas_root);
    p.local_box = std::move(local_box);
    p.blas_depth = blas_depth;
  }
  WideBvhHost w;
  w.nodes = std::move(node_words);
  w.tris = std::move(rec_floats);
  w.depth = depth;
  // emissive triangles, sampled uniformly over their total area
  std::vector<float4> em;
  std::vector<float> cdf;
  double total = 0.0;
  for (size_t t = 0; t < ntri && !two_level; ++t) {
    if (!mats[tri_mat[t]].emissive) continue;
    const float* a = &pos[4 * idx[4 * t]];
    const float* b = &pos[4 * idx[4 * t + 1]];
    const float* c = &pos[4 * idx[4 * t + 2]];
    const double e1[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
    const double e2[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
    const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                 cz = e1[0] * e2[1] - e1[1] * e2[0];
    const double area = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
    if (!(area > 0.0)) continue;
    uint32_t mb = tri_mat[t];
    float mf;
    std::memcpy(&mf, &mb, 4);
    em.push_back(make_float4(a[0], a[1], a[2], mf));
    em.push_back(make_float4(b[0], b[1], b[2], (float)area));
    em.push_back(make_float4(c[0], c[1], c[2], 0.0f));
    total += area;
    cdf.push_back((float)total);
  }
  for (float& x : cdf) x = (float)(x / total);
  if (!cdf.empty()) cdf.back() = 1.0f;
  // positional delta lights: points (inverse square, no range), then spots
  // (emitterPacking.ts:652-705: cos outer, cos inner = cos(angle (1 - penumbra)), range, decay)
  std::vector<float4> pts;
  auto finite3 = [](const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); };
  if (sc->point_light_count && !sc->point_lights) fail(VT_ERR_INVALID_ARGUMENT, "point_lights is null");
  for (size_t i = 0; i < sc->point_light_count; ++i) {
    const vt_point_light_desc& p = sc->point_lights[i];
    if (!finite3(p.position) || !finite3(p.intensity)) fail(VT_ERR_RANGE, "point light " + std::to_string(i) + " is not finite");
    pts.push_back(make_float4(p.position[0], p.position[1], p.position[2], 0.0f));
    pts.push_back(make_float4(p.intensity[0], p.intensity[1], p.intensity[2], 0.0f));
    pts.push_back(make_float4(0.0f, 0.0f, 0.0f, -2.0f));
    pts.push_back(make_float4(-1.0f, 0.0f, 2.0f, 0.0f));
  }
  if (sc->spot_light_count && !sc->spot_lights) fail(VT_ERR_INVALID_ARGUMENT, "spot_lights is null");
  for (size_t i = 0; i < sc->spot_light_count; ++i) {
    const vt_spot_light_desc& p = sc->spot_lights[i];
    const std::string who = "spot light " + std::to_string(i);
    if (!finite3(p.position) || !finite3(p.intensity) || !finite3(p.direction)) fail(VT_ERR_RANGE, who + " is not finite");
    const double dl = std::sqrt((double)p.direction[0] * p.direction[0] + (double)p.direction[1] * p.direction[1] +
                                (double)p.direction[2] * p.direction[2]);
    if (!(dl > 0.0)) fail(VT_ERR_INVALID_ARGUMENT, who + ": direction is zero");
    if (!(p.angle > 0.0f) || !(p.angle <= (float)M_PI)) fail(VT_ERR_RANGE, who + ": angle must be in (0, pi]");
    if (!(p.penumbra >= 0.0f && p.penumbra <= 1.0f)) fail(VT_ERR_RANGE, who + ": penumbra must be in [0, 1]");
    if (!(p.distance >= 0.0f) || !std::isfinite(p.distance)) fail(VT_ERR_RANGE, who + ": distance must be >= 0");
    if (!(p.decay >= 0.0f) || !std::isfinite(p.decay)) fail(VT_ERR_RANGE, who + ": decay must be >= 0");
    const double outer = p.angle, inner = outer * (1.0 - p.penumbra);
    pts.push_back(make_float4(p.position[0], p.position[1], p.position[2], 0.0f));
    pts.push_back(make_float4(p.intensity[0], p.intensity[1], p.intensity[2], 0.0f));
    pts.push_back(make_float4((float)(p.direction[0] / dl), (float)(p.direction[1] / dl), (float)(p.direction[2] / dl),
                              (float)std::cos(outer)));
    pts.push_back(make_float4((float)std::cos(inner), p.distance, p.decay, 1.0f));
  }
  // analytic area lights: rectangles, then discs (emitterPacking.ts:78-93: centre, half axes, radiance, shape)
  std::vector<float4> areas;
  if (sc->rect_light_count && !sc->rect_lights) fail(VT_ERR_INVALID_ARGUMENT, "rect_lights is null");
  for (size_t i = 0; i < sc->rect_light_count; ++i) {
    const vt_rect_light_desc& r = sc->rect_lights[i];
    const std::string who = "rect light " + std::to_string(i);
    if (!finite3(r.corner) || !finite3(r.edge_u) || !finite3(r.edge_v) || !finite3(r.radiance))
      fail(VT_ERR_RANGE, who + " is not finite");
    float c[3], u[3], v[3];
    for (int k = 0; k < 3; ++k) {
      u[k] = 0.5f * r.edge_u[k];
      v[k] = 0.5f * r.edge_v[k];
      c[k] = r.corner[k] + u[k] + v[k];
    }
    const double cx = (double)u[1] * v[2] - (double)u[2] * v[1], cy = (double)u[2] * v[0] - (double)u[0] * v[2],
                 cz = (double)u[0] * v[1] - (double)u[1] * v[0];
    const double area = 4.0 * std::sqrt(cx * cx + cy * cy + cz * cz);
    if (!(area > 0.0) || !std::isfinite(area)) fail(VT_ERR_INVALID_ARGUMENT, who + " has no area");
    areas.push_back(make_float4(c[0], c[1], c[2], 0.0f));
    areas.push_back(make_float4(u[0], u[1], u[2], (float)area));
    areas.push_back(make_float4(v[0], v[1], v[2], 0.0f));
    areas.push_back(make_float4(r.radiance[0], r.radiance[1], r.radiance[2], 0.0f));
  }
  if (sc->disc_light_count && !sc->disc_lights) fail(VT_ERR_INVALID_ARGUMENT, "disc_lights is null");
  for (size_t i = 0; i < sc->disc_light_count; ++i) {
    const vt_disc_light_desc& d = sc->disc_lights[i];
    const std::string who = "disc light " + std::to_string(i);
    if (!finite3(d.center) || !finite3(d.normal) || !finite3(d.radiance) || !std::isfinite(d.radius))
      fail(VT_ERR_RANGE, who + " is not finite");
    if (!(d.radius > 0.0f)) fail(VT_ERR_RANGE, who + ": radius must be > 0");
    const double nl = std::sqrt((double)d.normal[0] * d.normal[0] + (double)d.normal[1] * d.normal[1] +
                                (double)d.normal[2] * d.normal[2]);
    if (!(nl > 0.0)) fail(VT_ERR_INVALID_ARGUMENT, who + ": normal is zero");
    const double n[3] = {d.normal[0] / nl, d.normal[1] / nl, d.normal[2] / nl};
    // tangent frame (t, b) with t x b = n, scaled by the radius
    double t[3];
    if (std::fabs(n[0]) > 0.9) { t[0] = -n[2]; t[1] = 0.0; t[2] = n[0]; }
    else { t[0] = 0.0; t[1] = n[2]; t[2] = -n[1]; }
    const double tl = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    for (double& x : t) x /= tl;
    const double b[3] = {n[1] * t[2] - n[2] * t[1], n[2] * t[0] - n[0] * t[2], n[0] * t[1] - n[1] * t[0]};
    const double rr = d.radius;
    areas.push_back(make_float4(d.center[0], d.center[1], d.center[2], 1.0f));
    areas.push_back(make_float4((float)(t[0] * rr), (float)(t[1] * rr), (float)(t[2] * rr), (float)(M_PI * rr * rr)));
    areas.push_back(make_float4((float)(b[0] * rr), (float)(b[1] * rr), (float)(b[2] * rr), 0.0f));
    areas.push_back(make_float4(d.radiance[0], d.radiance[1], d.radiance[2], 0.0f));
  }
  // directional lights
  std::vector<float4> dirs;
  if (sc->directional_light_count && !sc->directional_lights) fail(VT_ERR_INVALID_ARGUMENT, "directional_lights is null");
  for (size_t i = 0; i < sc->directional_light_count; ++i) {
    const vt_directional_light_desc& dl = sc->directional_lights[i];
    const double dx = dl.direction[0], dy = dl.direction[1], dz = dl.direction[2];
    const double len = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (!(len > 0.0) || !std::isfinite(len)) fail(VT_ERR_INVALID_ARGUMENT, "directional light direction is zero");
    if (!(dl.angular_radius >= 0.0f) || !(dl.angular_radius < 1.5f))
      fail(VT_ERR_RANGE, "directional light angular_radius must be in [0, 1.5)");
    const bool delta = dl.angular_radius == 0.0f;
    const double st = std::sin((double)dl.angular_radius);
    const double to_l = delta ? 1.0 : 1.0 / (M_PI * st * st);  // disc radiance from its irradiance
    dirs.push_back(make_float4((float)(-dx / len), (float)(-dy / len), (float)(-dz / len),
                               delta ? 1.0f : (float)std::cos((double)dl.angular_radius)));
    dirs.push_back(make_float4((float)(dl.irradiance[0] * to_l), (float)(dl.irradiance[1] * to_l),
                               (float)(dl.irradiance[2] * to_l), delta ? 1.0f : 0.0f));
  }
  // environment: equirectangular, importance by luminance * sin(theta)
  std::vector<float4> envt;
  std::vector<float> marg, cond;
  const bool has_env = sc->environment_rgb && sc->environment_width > 0 && sc->environment_height > 0;
  bool env_sampleable = false;
  double env_total = 0.0;  // sum of luminance * intensity * sin(theta) over the texels
  if (has_env) {
    const int W = sc->environment_width, H = sc->environment_height;
    const float scale = sc->environment_intensity > 0.0f ? sc->environment_intensity : 1.0f;
    envt.resize((size_t)W * H);
    cond.resize((size_t)H * (W + 1));
    marg.resize(H + 1);
    std::vector<double> rows(H);
    double tot = 0.0;
    for (int r = 0; r < H; ++r) {
      const double st = std::sin(M_PI * (r + 0.5) / H);
      double acc = 0.0;
      cond[(size_t)r * (W + 1)] = 0.0f;
      std::vector<double> cum(W);
      for (int c = 0; c < W; ++c) {
        const float* px = sc->environment_rgb + 3 * ((size_t)r * W + c);
        envt[(size_t)r * W + c] = make_float4(px[0], px[1], px[2], 0.0f);
        acc += std::max(0.0, luminance(px) * scale) * st;
        cum[c] = acc;
      }
      for (int c = 0; c < W; ++c) cond[(size_t)r * (W + 1) + c + 1] = acc > 0 ? (float)(cum[c] / acc) : (float)(c + 1) / W;
      cond[(size_t)r * (W + 1) + W] = 1.0f;
      rows[r] = acc;
      tot += acc;
    }
    marg[0] = 0.0f;
    double run = 0.0;
    for (int r = 0; r < H; ++r) {
      run += rows[r];
      marg[r + 1] = tot > 0 ? (float)(run / tot) : (float)(r + 1) / H;
    }
    marg[H] = 1.0f;
    env_sampleable = tot > 0.0;
    env_total = tot;
  }
  // light tree over the positional light entries, in sample_light's order: the
  // emissive-mesh group, points, spots, rectangles, discs (the reference's
  // buildLightTreeInputForScene, emitterPacking.ts:1005-1232, with the emissive
  // triangles as one entry sampled by area)
  {
    std::vector<lt::Emitter> le;
    auto lum_f = [](double r, double g, double b) { return (double)(float)(0.2126 * r + 0.7152 * g + 0.0722 * b); };
    auto unit = [](const double* v, double* o) {
      const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      for (int k = 0; k < 3; ++k) o[k] = l > 1e-12 ? v[k] / l : 0.0;
    };
    if (!em.empty()) {
      lt::Emitter g;
      for (int k = 0; k < 3; ++k) { g.mn[k] = INFINITY; g.mx[k] = -INFINITY; }
      std::vector<lt::Emitter> tris(em.size() / 3);
      for (size_t k = 0; k < tris.size(); ++k) {
        const float4 a = em[3 * k], b = em[3 * k + 1], c = em[3 * k + 2];
        uint32_t mb;
        std::memcpy(&mb, &a.w, 4);
        const float3 L = mats[mb].emission;
        g.power += (double)(float)(lum_f(L.x, L.y, L.z) * (double)b.w);
        const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z}, C[3] = {c.x, c.y, c.z};
        for (int q = 0; q < 3; ++q) {
          g.mn[q] = std::min(g.mn[q], std::min(A[q], std::min(B[q], C[q])));
          g.mx[q] = std::max(g.mx[q], std::max(A[q], std::max(B[q], C[q])));
        }
        const double e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]}, e2[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
        const double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        tris[k].oriented = true;
        unit(n, tris[k].axis);
      }
      for (int k = 0; k < 3; ++k) g.centroid[k] = 0.5 * g.mn[k] + 0.5 * g.mx[k];
      // one-sided emitters: the group's cone bounds every triangle's outward hemisphere
      lt::merge_into(g, tris);
      le.push_back(g);
    }
    for (size_t i = 0; i < pts.size() / pt::kPositionalF4; ++i) {
      const float4* q = &pts[pt::kPositionalF4 * i];
      const float4 P = q[0], I = q[1], ax = q[2];
      lt::Emitter e;
      e.power = lum_f(I.x, I.y, I.z);
      const double c[3] = {P.x, P.y, P.z};
      for (int k = 0; k < 3; ++k) e.centroid[k] = e.mn[k] = e.mx[k] = c[k];
      if (q[3].w != 0.0f) {  // spot: its beam
        e.oriented = true;
        const double a[3] = {ax.x, ax.y, ax.z};
        unit(a, e.axis);
        e.theta_o = 0.0;
        e.theta_e = std::acos(std::max(-1.0, std::min(1.0, (double)ax.w)));
      }
      le.push_back(e);
    }
    for (size_t i = 0; i < areas.size() / pt::kAreaLightF4; ++i) {
      const float4* q = &areas[pt::kAreaLightF4 * i];
      const float4 c = q[0], u = q[1], v = q[2], L = q[3];
      lt::Emitter e;
      e.power = (double)(float)(lum_f(L.x, L.y, L.z) * (double)u.w);
      const double C[3] = {c.x, c.y, c.z}, U[3] = {u.x, u.y, u.z}, W[3] = {v.x, v.y, v.z};
      const double r = std::sqrt(U[0] * U[0] + U[1] * U[1] + U[2] * U[2]);
      for (int k = 0; k < 3; ++k) {
        const double h = c.w != 0.0f ? r : std::fabs(U[k]) + std::fabs(W[k]);
        e.centroid[k] = C[k];
        e.mn[k] = C[k] - h;
        e.mx[k] = C[k] + h;
      }
      const double n[3] = {U[1] * W[2] - U[2] * W[1], U[2] * W[0] - U[0] * W[2], U[0] * W[1] - U[1] * W[0]};
      e.oriented = true;
      unit(n, e.axis);
      le.push_back(e);
    }
    // the distant entries (directionals, the environment) are chosen outside the
    // tree, evenly within n_dist / (n_dist + 1) of the selection (light_tree.cuh)
    if (le.size() >= 2) p.light_tree = lt::build_packed(le);
  }
  if (two_level && (node_base || rec_base)) fail(VT_ERR_INVALID_ARGUMENT, "instanced scenes cannot be offset");
  p.two_level = two_level;
  p.node_words = std::move(w.nodes);
  p.rec_floats = std::move(w.tris);
  p.depth = w.depth;
  p.stack_depth = two_level ? 2 * w.depth + 6 : 2 * w.depth + 2;
  if (p.stack_depth > kTraversalStack)
    fail(VT_ERR_BUILD, "8-wide encoding proof: traversal needs " + std::to_string(p.stack_depth) +
                           " stack entries (top and bottom levels), capacity " + std::to_string(kTraversalStack));
  p.root = two_level ? root : node_base;
  p.inst_lanes = std::move(inst_lanes);
  p.inst_tab = std::move(inst_tab);
  p.inst_rows = std::move(inst_rows);
  p.n_instances = sc->instance_count;
  p.mats = std::move(mats);
  p.emitters = std::move(em);
  p.cdf = std::move(cdf);
  p.emit_total = total;
  p.points = std::move(pts);
  p.area_lights = std::move(areas);
  p.dirs = std::move(dirs);
  p.env = std::move(envt);
  p.marg = std::move(marg);
  p.cond = std::move(cond);
  p.has_env = has_env;
  p.env_sampleable = env_sampleable;
  p.env_w = has_env ? sc->environment_width : 0;
  p.env_h = has_env ? sc->environment_height : 0;
  p.env_scale = sc->environment_intensity > 0.0f ? sc->environment_intensity : 1.0f;
  if (!std::isfinite(sc->environment_rotation_y)) fail(VT_ERR_RANGE, "environment_rotation_y is not finite");
  p.env_rotation = sc->environment_rotation_y;
  p.ntri = ntri;
  return p;
}

}  // namespace vt
