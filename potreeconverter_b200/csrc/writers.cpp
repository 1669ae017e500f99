// hierarchy.bin and metadata.json writers. Both files are byte contracts
// with the reference's readers (Potree), so their layout follows the
// reference writers step for step, including its quirks:
//  * every node starts as LEAF and only turns NORMAL when one of its children
//    is met later in the same batch (HierarchyBuilder.h:149-163); since
//    children complete before parents, inner nodes keep type LEAF with a
//    non-zero child mask;
//  * batch roots are PROXY in the root batch and NORMAL inside their own
//    batch (HierarchyBuilder.h:257-264, 316-327);
//  * byte sizes pass through a 32-bit field (indexer.h:221, HierarchyBuilder.h:104).

#include "writers.h"

#include <algorithm>
#include <iomanip>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <unordered_map>

namespace pcg {

namespace {

constexpr int kStep = 4;           // hierarchyStepSize, indexer.cpp:19
constexpr int kRecordBytes = 22;   // type, childMask, numPoints, offset, size

enum NodeType : uint8_t { T_NORMAL = 0, T_LEAF = 1, T_PROXY = 2 };

struct BNode {
	std::string name;
	int32_t num_points = 0;
	uint8_t child_mask = 0;
	uint64_t byte_offset = 0, byte_size = 0;
	uint8_t type = T_LEAF;
	uint64_t proxy_offset = 0, proxy_size = 0;
};

struct BChunk {
	std::string name;
	std::vector<BNode*> nodes;
	int64_t byte_offset = 0;
};

struct Batch {
	std::string name;
	std::vector<std::unique_ptr<BNode>> nodes;
	std::vector<std::unique_ptr<BChunk>> chunks;
	std::unordered_map<std::string, BNode*> node_of;
	std::unordered_map<std::string, BChunk*> chunk_of;
	int64_t byte_size = 0;
};

bool bfs_less(const std::string& a, const std::string& b) {
	return a.size() != b.size() ? a.size() < b.size() : a < b;
}

BChunk* chunk_for(Batch& b, const std::string& key) {
	auto it = b.chunk_of.find(key);
	if (it != b.chunk_of.end()) return it->second;
	b.chunks.push_back(std::make_unique<BChunk>());
	b.chunks.back()->name = key;
	b.chunk_of[key] = b.chunks.back().get();
	return b.chunks.back().get();
}

// HierarchyBuilder::loadBatch (HierarchyBuilder.h:82-197) over the records a
// flusher file holds, in file order.
std::unique_ptr<Batch> load_batch(const std::string& name, const std::vector<const HierRecord*>& recs) {
	auto b = std::make_unique<Batch>();
	b->name = name;
	for (const HierRecord* r : recs) {
		auto n = std::make_unique<BNode>();
		n->name = r->name;
		n->num_points = (int32_t)(uint32_t)r->num_points;
		n->byte_offset = (uint64_t)r->byte_offset;
		n->byte_size = (uint64_t)(int64_t)(int32_t)(uint32_t)r->byte_size;
		// chunk key: "r" for names up to 5 chars, then the first 4k+1 chars
		size_t len = n->name.size();
		std::string key = len <= 5 ? n->name.substr(0, 1) : n->name.substr(0, kStep * ((len - 2) / 4) + 1);
		if (n->name == b->name) key = n->name;
		BNode* np = n.get();
		chunk_for(*b, key)->nodes.push_back(np);
		b->node_of[np->name] = np;
		b->nodes.push_back(std::move(n));
		if ((len - 1) % kStep == 0 && len > (size_t)kStep + 1) chunk_for(*b, np->name)->nodes.push_back(np);
	}
	std::sort(b->chunks.begin(), b->chunks.end(), [](const auto& x, const auto& y) { return bfs_less(x->name, y->name); });
	for (auto& n : b->nodes) {
		n->type = T_LEAF;
		auto it = b->node_of.find(n->name.substr(0, n->name.size() - 1));
		if (it != b->node_of.end()) {
			it->second->type = T_NORMAL;
			it->second->child_mask |= (uint8_t)(1 << (n->name.back() - '0'));
		}
	}
	for (auto& c : b->chunks) {
		auto it = b->node_of.find(c->name);
		if (it != b->node_of.end()) it->second->type = T_PROXY;
	}
	for (auto& c : b->chunks)
		std::sort(c->nodes.begin(), c->nodes.end(), [](const BNode* x, const BNode* y) { return bfs_less(x->name, y->name); });
	return b;
}

bool process_batch(Batch& b, std::string& err) {  // HierarchyBuilder.h:199-238
	int64_t off = 0;
	for (auto& c : b.chunks) {
		c->byte_offset = off;
		if (c->name != b.name) {
			std::string parent = c->name.substr(0, c->name.size() - kStep);
			if (!b.chunk_of.count(parent)) { err = "hierarchy: missing parent chunk " + parent; return false; }
			auto it = b.node_of.find(c->name);
			if (it == b.node_of.end()) { err = "hierarchy: missing proxy node " + c->name; return false; }
			it->second->type = T_PROXY;
			it->second->proxy_offset = (uint64_t)c->byte_offset;
			it->second->proxy_size = (uint64_t)kRecordBytes * c->nodes.size();
		}
		off += kRecordBytes * (int64_t)c->nodes.size();
	}
	b.byte_size = off;
	return true;
}

void serialize_batch(Batch& b, int64_t bytes_written, std::vector<uint8_t>& out, size_t at) {  // :240-282
	size_t k = 0;
	size_t total = 0;
	for (auto& c : b.chunks) total += c->nodes.size();
	if (out.size() < at + kRecordBytes * total) out.resize(at + kRecordBytes * total);
	for (auto& c : b.chunks) {
		for (BNode* n : c->nodes) {
			bool is_proxy = n->type == T_PROXY && n->name != c->name;
			uint8_t type = (n->type == T_PROXY && !is_proxy) ? (uint8_t)T_NORMAL : n->type;
			uint64_t size = is_proxy ? n->proxy_size : n->byte_size;
			uint64_t offset = is_proxy ? (uint64_t)bytes_written + n->proxy_offset : n->byte_offset;
			uint32_t np = (uint32_t)n->num_points;
			uint8_t* p = out.data() + at + kRecordBytes * k;
			p[0] = type;
			p[1] = n->child_mask;
			std::memcpy(p + 2, &np, 4);
			std::memcpy(p + 6, &offset, 8);
			std::memcpy(p + 14, &size, 8);
			k++;
		}
	}
	b.byte_size = (int64_t)(kRecordBytes * total);
}

}  // namespace

bool build_hierarchy(const std::vector<HierRecord>& completed, std::vector<uint8_t>& out,
                     int64_t& first_chunk_size, std::string& err) {
	// flusher files: per key, records in completion order (indexer.h:171-193);
	// the builder visits files in file-name order, which equals key order.
	std::map<std::string, std::vector<const HierRecord*>> files;
	for (const auto& r : completed) {
		const std::string key = r.name.size() <= (size_t)kStep + 1 ? std::string("r") : r.name.substr(0, kStep + 1);
		files[key].push_back(&r);
		if (r.name.size() == (size_t)kStep + 1) files[r.name].push_back(&r);
	}
	auto rit = files.find("r");
	if (rit == files.end()) { err = "hierarchy: no root batch"; return false; }
	auto root = load_batch("r", rit->second);
	out.assign(kRecordBytes * root->nodes.size(), 0);
	int64_t written = (int64_t)out.size();
	for (auto& [key, recs] : files) {
		if (key == "r") continue;
		auto b = load_batch(key, recs);
		if (!process_batch(*b, err)) return false;
		size_t at = out.size();
		serialize_batch(*b, written, out, at);
		auto pit = root->node_of.find(b->name);
		if (pit == root->node_of.end()) { err = "hierarchy: batch root missing from root batch"; return false; }
		if (b->nodes.size() > 1) {
			pit->second->type = T_PROXY;
			pit->second->proxy_offset = (uint64_t)written;
			pit->second->proxy_size = (uint64_t)kRecordBytes * b->chunk_of[b->name]->nodes.size();
		} else {
			pit->second->type = T_LEAF;
		}
		written += b->byte_size;
	}
	std::vector<uint8_t> head;
	serialize_batch(*root, 0, head, 0);
	std::memcpy(out.data(), head.data(), head.size());
	first_chunk_size = root->byte_size;
	return true;
}

std::string build_metadata(const std::string& name, const std::string& projection, int64_t points_total,
                           int64_t first_chunk_size, int64_t depth, const Setup& s,
                           const std::vector<AttrStats>& stats, double spacing) {
	auto num = [](double v) {
		std::ostringstream o;
		o << std::setprecision(std::numeric_limits<double>::max_digits10) << v;
		return o.str();
	};
	auto q = [](const std::string& v) { return "\"" + v + "\""; };
	auto tabs = [](int n) { return std::string(n, '\t'); };
	auto vec3 = [&](const Vec3d& v) { return "[" + num(v.x) + ", " + num(v.y) + ", " + num(v.z) + "]"; };
	auto list = [&](std::initializer_list<double> vs) {
		std::string o = "[";
		size_t i = 0;
		for (double v : vs) { o += num(v); if (++i < vs.size()) o += ", "; }
		return o + "]";
	};
	std::ostringstream m;
	const char* nl = "\n";
	m << "{" << nl;
	m << tabs(1) << q("version") << ": " << q("2.0") << "," << nl;
	m << tabs(1) << q("name") << ": " << q(name) << "," << nl;
	m << tabs(1) << q("description") << ": " << q("") << "," << nl;
	m << tabs(1) << q("points") << ": " << points_total << "," << nl;
	m << tabs(1) << q("projection") << ": " << q(projection) << "," << nl;
	m << tabs(1) << q("hierarchy") << ": {" << nl;
	m << tabs(2) << q("firstChunkSize") << ": " << first_chunk_size << ", " << nl;
	m << tabs(2) << q("stepSize") << ": " << kStep << ", " << nl;
	m << tabs(2) << q("depth") << ": " << depth << nl;
	m << tabs(1) << "}," << nl;
	m << tabs(1) << q("offset") << ": " << vec3(s.pos_offset) << "," << nl;
	m << tabs(1) << q("scale") << ": " << vec3(s.pos_scale) << "," << nl;
	m << tabs(1) << q("spacing") << ": " << num(spacing) << "," << nl;
	m << tabs(1) << q("boundingBox") << ": {" << nl;
	m << tabs(2) << q("min") << ": " << vec3(s.cube_min) << ", " << nl;
	m << tabs(2) << q("max") << ": " << vec3(s.root_max) << nl;
	m << tabs(1) << "}," << nl;
	m << tabs(1) << q("encoding") << ": " << q("DEFAULT") << "," << nl;
	m << tabs(1) << q("attributes") << ": [" << nl;
	for (size_t i = 0; i < s.attrs.size(); i++) {
		const AttrDesc& a = s.attrs[i];
		const AttrStats& st = stats[i];
		if (i == 0) m << tabs(2) << "{" << nl;
		m << tabs(3) << q("name") << ": " << q(a.name) << "," << nl;
		m << tabs(3) << q("description") << ": " << q(a.description) << "," << nl;
		m << tabs(3) << q("size") << ": " << a.size << "," << nl;
		m << tabs(3) << q("numElements") << ": " << a.numElements << "," << nl;
		m << tabs(3) << q("elementSize") << ": " << a.elementSize << "," << nl;
		m << tabs(3) << q("type") << ": " << q(attr_type_name(a.type)) << "," << nl;
		bool any = false;
		for (int64_t h : st.histogram) any = any || h != 0;
		if (a.size == 1 && any) {
			m << tabs(3) << q("histogram") << ": [";
			for (size_t k = 0; k < st.histogram.size(); k++) { m << st.histogram[k]; if (k + 1 < st.histogram.size()) m << ", "; }
			m << "], " << nl;
		}
		if (a.numElements == 1) {
			m << tabs(3) << q("min") << ": " << list({st.min.x}) << "," << nl;
			m << tabs(3) << q("max") << ": " << list({st.max.x}) << "," << nl;
			m << tabs(3) << q("scale") << ": " << list({a.scale.x}) << "," << nl;
			m << tabs(3) << q("offset") << ": " << list({a.offset.x}) << nl;
		} else if (a.numElements == 2) {
			m << tabs(3) << q("min") << ": " << list({st.min.x, st.min.y}) << "," << nl;
			m << tabs(3) << q("max") << ": " << list({st.max.x, st.max.y}) << "," << nl;
			m << tabs(3) << q("scale") << ": " << list({a.scale.x, a.scale.y}) << "," << nl;
			m << tabs(3) << q("offset") << ": " << list({a.offset.x, a.offset.y}) << nl;
		} else if (a.numElements == 3) {
			m << tabs(3) << q("min") << ": " << list({st.min.x, st.min.y, st.min.z}) << "," << nl;
			m << tabs(3) << q("max") << ": " << list({st.max.x, st.max.y, st.max.z}) << "," << nl;
			m << tabs(3) << q("scale") << ": " << list({a.scale.x, a.scale.y, a.scale.z}) << "," << nl;
			m << tabs(3) << q("offset") << ": " << list({a.offset.x, a.offset.y, a.offset.z}) << nl;
		}
		m << tabs(2) << (i + 1 < s.attrs.size() ? "},{" : "}") << nl;
	}
	m << tabs(1) << "]" << nl;
	m << "}" << nl;
	return m.str();
}

}  // namespace pcg
