// ref_bvh_harness.cpp -- TEST INFRASTRUCTURE ONLY (oracle).
//
// A thin C-ABI harness around the reference renderer's own BVH template
// (src/Library/Acceleration/BVH.h) and its double-precision ray/triangle
// test (src/Library/Intersection/RayTriangleIntersection.cpp:21-68).  The
// recipe in oracle/Makefile compiles this file together with those reference
// sources where they lie (they are never copied into this repository) into
// oracle/_ref/libref_bvh.so.
//
// The element type is a plain triangle index (uint32_t).  The element
// processor below restates the triangle-mesh leaf processor of the reference
// (src/Library/Geometry/TriangleMeshGeometryIndexedSpecializations.h:116-525)
// minus the shading attributes it does not need, and records the index of the
// closest accepted triangle, because the reference hit record carries no
// primitive id (src/Library/Intersection/RayIntersectionGeometric.h:87-90).
//
// Only tests, the smoke check and bench.py's CPU-baseline leg may load this.

#include "Acceleration/BVH.h"
#include "Intersection/RayPrimitiveIntersections.h"
#include "Interfaces/ILog.h"
#include "Interfaces/IOptions.h"

#include <cstdarg>
#include <cstdio>
#include <thread>
#include <vector>
#include <atomic>

namespace RISE
{
	// Quiet logger: the BVH template prints build statistics through
	// GlobalLog(); the harness does not link the reference's log subsystem.
	class QuietLog : public ILog
	{
	public:
		void Print( LOG_ENUM, const char* ) const override {}
		void PrintEx( LOG_ENUM, const char*, ... ) const override {}
		void PrintNew( const void*, const char*, const int, const char* ) const override {}
		void PrintNew( const IReference*, const char*, const int, const char* ) const override {}
		void PrintDelete( const void*, const char*, const int ) const override {}
		void PrintDelete( const IReference*, const char*, const int ) const override {}
		void FlushPrinters() override {}
	};
	ILog* GlobalLog() { static QuietLog log; return &log; }
	void GlobalLogCleanupAndShutdown() {}

	// Default-valued options: the reference's thread wrapper reads one
	// scheduling option; the harness does not link the options-file parser.
	class DefaultOptions : public IOptions
	{
	public:
		void addref() const override {}
		bool release() const override { return false; }
		unsigned int refcount() const override { return 1; }
		int ReadInt( const char*, int d ) override { return d; }
		double ReadDouble( const char*, double d ) override { return d; }
		bool ReadBool( const char*, bool d ) override { return d; }
		String ReadString( const char*, String d ) override { return d; }
	};
	IOptions& GlobalOptions() { static DefaultOptions o; return o; }
}

using namespace RISE;

namespace
{
	thread_local int32_t g_lastHit = -1;

	struct TriProcessor : public TreeElementProcessor<uint32_t>
	{
		const double* v;   // 9 doubles per triangle (v0, v1, v2)

		void addref() const override {}
		bool release() const override { return false; }
		unsigned int refcount() const override { return 1; }

		inline void Verts( uint32_t t, Point3& a, Point3& b, Point3& c ) const
		{
			const double* p = v + 9ull * t;
			a = Point3( p[0], p[1], p[2] );
			b = Point3( p[3], p[4], p[5] );
			c = Point3( p[6], p[7], p[8] );
		}

		void RayElementIntersection( RayIntersectionGeometric& ri, const uint32_t elem,
			const bool bHitFrontFaces, const bool bHitBackFaces ) const override
		{
			Point3 a, b, c; Verts( elem, a, b, c );
			const Vector3 ea = Vector3Ops::mkVector3( b, a );
			const Vector3 eb = Vector3Ops::mkVector3( c, a );
			const Vector3 fn = Vector3Ops::Cross( ea, eb );
			if( !bHitFrontFaces && Vector3Ops::Dot( fn, ri.ray.Dir() ) < 0 ) return;
			if( !bHitBackFaces && Vector3Ops::Dot( fn, ri.ray.Dir() ) > 0 ) return;
			TRIANGLE_HIT h;
			h.bHit = false;
			h.dRange = RISE_INFINITY;
			RayTriangleIntersection( ri.ray, h, a, ea, eb );
			if( h.bHit && h.dRange < ri.range ) {
				ri.bHit = true;
				ri.range = h.dRange;
				g_lastHit = (int32_t)elem;
			}
		}
		void RayElementIntersection( RayIntersection& ri, const uint32_t elem,
			const bool f, const bool b, const bool ) const override
		{
			RayElementIntersection( ri.geometric, elem, f, b );
		}
		bool RayElementIntersection_IntersectionOnly( const Ray& ray, const Scalar dHowFar,
			const uint32_t elem, const bool bHitFrontFaces, const bool bHitBackFaces ) const override
		{
			Point3 a, b, c; Verts( elem, a, b, c );
			const Vector3 ea = Vector3Ops::mkVector3( b, a );
			const Vector3 eb = Vector3Ops::mkVector3( c, a );
			const Vector3 fn = Vector3Ops::Cross( ea, eb );
			if( !bHitFrontFaces && Vector3Ops::Dot( fn, ray.Dir() ) < 0 ) return false;
			if( !bHitBackFaces && Vector3Ops::Dot( fn, ray.Dir() ) > 0 ) return false;
			TRIANGLE_HIT h;
			RayTriangleIntersection( ray, h, a, ea, eb );
			return h.bHit && ( h.dRange > NEARZERO && h.dRange < dHowFar );
		}
		BoundingBox GetElementBoundingBox( const uint32_t elem ) const override
		{
			BoundingBox bb( Point3( RISE_INFINITY, RISE_INFINITY, RISE_INFINITY ),
			                Point3( -RISE_INFINITY, -RISE_INFINITY, -RISE_INFINITY ) );
			Point3 a, b, c; Verts( elem, a, b, c );
			bb.Include( a ); bb.Include( b ); bb.Include( c );
			return bb;
		}
		bool ElementBoxIntersection( const uint32_t, const BoundingBox& ) const override { return true; }
		char WhichSideofPlaneIsElement( const uint32_t, const Plane& ) const override { return 0; }
		void SerializeElement( IWriteBuffer&, const uint32_t ) const override {}
		void DeserializeElement( IReadBuffer&, uint32_t& ) const override {}
		bool GetFloatTriangleVertices( const uint32_t elem, float a[3], float b[3], float c[3] ) const override
		{
			const double* p = v + 9ull * elem;
			for( int k = 0; k < 3; ++k ) { a[k] = (float)p[k]; b[k] = (float)p[3 + k]; c[k] = (float)p[6 + k]; }
			return true;
		}
	};

	// Subclass only to read the protected node arrays for export.
	class ExportBVH : public BVH<uint32_t>
	{
	public:
		ExportBVH( const TreeElementProcessor<uint32_t>& ep, const std::vector<uint32_t>& prims,
		           const BoundingBox& hint, const AccelerationConfig& cfg )
			: BVH<uint32_t>( ep, prims, hint, cfg ) {}
		const std::vector<Node>& Nodes2() const { return nodes; }
		const std::vector<uint32_t>& Prims() const { return prims; }
		const std::vector<BVH4Node>& Nodes4() const { return nodes4; }
	};

	struct Handle
	{
		std::vector<double> verts;
		TriProcessor proc;
		ExportBVH* bvh = nullptr;
	};

	template< class F >
	void ParallelRange( int64_t n, int threads, F fn )
	{
		if( threads <= 1 || n < 1024 ) { fn( 0, n ); return; }
		std::atomic<int64_t> next( 0 );
		const int64_t chunk = 4096;
		std::vector<std::thread> pool;
		for( int t = 0; t < threads; ++t ) {
			pool.emplace_back( [&]() {
				for( ;; ) {
					const int64_t s = next.fetch_add( chunk );
					if( s >= n ) break;
					fn( s, std::min( n, s + chunk ) );
				}
			} );
		}
		for( auto& th : pool ) th.join();
	}
}

extern "C" {

// Builds the reference BVH (leaf 4, 32 bins, Ctrav = Cint = 1 -- the
// triangle-mesh configuration at Geometry/TriangleMeshGeometryIndexed.cpp:529-535)
// over n_tri triangles given as 9 floats each.
void* ref_bvh_build( const float* tri9, int64_t n_tri )
{
	Handle* h = new Handle();
	h->verts.assign( tri9, tri9 + 9 * n_tri );
	h->proc.v = h->verts.data();
	std::vector<uint32_t> prims( (size_t)n_tri );
	for( int64_t i = 0; i < n_tri; ++i ) prims[(size_t)i] = (uint32_t)i;
	AccelerationConfig cfg;
	cfg.maxLeafSize = 4;
	cfg.binCount = 32;
	cfg.sahTraversalCost = 1.0;
	cfg.sahIntersectionCost = 1.0;
	cfg.doubleSided = true;
	BoundingBox hint( Point3( 0, 0, 0 ), Point3( 0, 0, 0 ) );
	h->bvh = new ExportBVH( h->proc, prims, hint, cfg );
	return h;
}

void ref_bvh_destroy( void* p )
{
	Handle* h = (Handle*)p;
	if( !h ) return;
	h->bvh->release();
	delete h;
}

int64_t ref_bvh_num_nodes2( void* p ) { return (int64_t)( (Handle*)p )->bvh->Nodes2().size(); }
int64_t ref_bvh_num_nodes4( void* p ) { return (int64_t)( (Handle*)p )->bvh->Nodes4().size(); }

// Copies the BVH2 nodes (32 bytes each, the reference's packed Node layout)
// and the reordered primitive indices.
void ref_bvh_export( void* p, void* nodes2_out, uint32_t* prims_out )
{
	Handle* h = (Handle*)p;
	const auto& n2 = h->bvh->Nodes2();
	if( !n2.empty() ) std::memcpy( nodes2_out, n2.data(), n2.size() * 32 );
	const auto& pr = h->bvh->Prims();
	if( !pr.empty() ) std::memcpy( prims_out, pr.data(), pr.size() * 4 );
}

// Copies the collapsed BVH4 nodes (128 bytes each).
void ref_bvh_export4( void* p, void* nodes4_out )
{
	Handle* h = (Handle*)p;
	const auto& n4 = h->bvh->Nodes4();
	if( !n4.empty() ) std::memcpy( nodes4_out, n4.data(), n4.size() * 128 );
}

// Closest hit through the reference traversal.  rays: 8 floats per ray
// (ox, oy, oz, tmin, dx, dy, dz, tmax); tmin/tmax are ignored (the reference
// closest-hit query has an unbounded range).  Writes the hit triangle index
// (-1 on miss) and the double-precision parametric distance.
void ref_closest( void* p, const float* rays, int64_t n, int32_t* id_out, double* t_out, int threads )
{
	Handle* h = (Handle*)p;
	ParallelRange( n, threads, [&]( int64_t s, int64_t e ) {
		for( int64_t i = s; i < e; ++i ) {
			const float* r = rays + 8 * i;
			Ray ray( Point3( r[0], r[1], r[2] ), Vector3( r[4], r[5], r[6] ) );
			RayIntersectionGeometric ri( ray, nullRasterizerState );
			g_lastHit = -1;
			h->bvh->IntersectRay( ri, true, true );
			id_out[i] = ri.bHit ? g_lastHit : -1;
			t_out[i] = ri.bHit ? ri.range : -1.0;
		}
	} );
}

// Any hit (shadow query) through the reference traversal, within (0, tmax).
void ref_any( void* p, const float* rays, int64_t n, uint8_t* occ_out, int threads )
{
	Handle* h = (Handle*)p;
	ParallelRange( n, threads, [&]( int64_t s, int64_t e ) {
		for( int64_t i = s; i < e; ++i ) {
			const float* r = rays + 8 * i;
			Ray ray( Point3( r[0], r[1], r[2] ), Vector3( r[4], r[5], r[6] ) );
			occ_out[i] = h->bvh->IntersectRay_IntersectionOnly( ray, (double)r[7], true, true ) ? 1 : 0;
		}
	} );
}

// The reference's double Moller-Trumbore on one triangle (known-answer tests).
int ref_ray_triangle( const double* o, const double* d, const double* v0,
                      const double* ea, const double* eb, double* t, double* alpha, double* beta )
{
	Ray ray( Point3( o[0], o[1], o[2] ), Vector3( d[0], d[1], d[2] ) );
	TRIANGLE_HIT hit;
	RayTriangleIntersection( ray, hit, Point3( v0[0], v0[1], v0[2] ),
		Vector3( ea[0], ea[1], ea[2] ), Vector3( eb[0], eb[1], eb[2] ) );
	*t = hit.dRange; *alpha = hit.alpha; *beta = hit.beta;
	return hit.bHit ? 1 : 0;
}

}
