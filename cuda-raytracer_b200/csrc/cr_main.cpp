// `cr` command line, the drop-in for the reference's CLI (src/cr.cu:9-68):
//   cr <scene.json> [-o a.png] [-s spp] [--resolution=WxH] [-k Radiance]
//      [-t tracer] [-a allocator] [--pfm out.pfm] [-l] [-h]
// Defaults as in the reference: a.png, 1 spp, 1024x768.  Unlike the
// reference, -k and -t are honoured (the reference parses and ignores them)
// and errors give a non-zero exit code.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/cr.h"

static void usage()
{
	std::printf(
		"Ray tracer for heterogeneous systems (B200 wavefront build)\n"
		"Usage: cr <scene.json> [options]\n"
		"  -o <file>            Place the output into <file>. (a.png)\n"
		"  -s, --sample-per-pixel <n>  Number of sample points per pixel. (1)\n"
		"  --resolution=<WxH>   Target resolution. (1024x768)\n"
		"  -k, --kernel <name>  Kernel function: Radiance, Normal, Visibility, HalfVector. (Radiance)\n"
		"  -t, --tracer <name>  Tracer. (CudaWavefront)\n"
		"  -a, --allocator <n>  Accepted for compatibility; device memory is managed internally.\n"
		"  --pfm <file>         Also write linear radiance as a PFM.\n"
		"  -l, --list           List kernels and tracers.\n"
		"  -v, --visualize      Not available (no graphics stack).\n"
		"  -h, --help           Show help message.\n" );
}

int main( int argc, char **argv )
{
	std::string scene, out = "a.png", res = "1024x768", kernel = "Radiance", tracer = "CudaWavefront", pfm;
	unsigned spp = 1;
	for ( int i = 1; i < argc; ++i )
	{
		std::string a = argv[ i ];
		auto val = [&]( const char *name ) -> std::string {
			size_t eq = a.find( '=' );
			if ( eq != std::string::npos ) return a.substr( eq + 1 );
			if ( i + 1 >= argc )
			{
				std::fprintf( stderr, "missing value for %s\n", name );
				std::exit( 2 );
			}
			return argv[ ++i ];
		};
		auto is = [&]( const char *s, const char *l ) {
			return a == s || a == l || ( a.rfind( std::string( l ) + "=", 0 ) == 0 ) ||
				   ( std::strlen( s ) == 2 && a.size() > 2 && a.rfind( s, 0 ) == 0 && a[ 2 ] != '-' );
		};
		if ( a == "-h" || a == "--help" )
		{
			usage();
			return 0;
		}
		else if ( a == "-l" || a == "--list" )
		{
			std::printf( "kernels: Radiance Normal Visibility HalfVector\ntracers: CudaWavefront (also accepts CPUMulticore)\n" );
			return 0;
		}
		else if ( a == "-v" || a == "--visualize" )
		{
			std::fprintf( stderr, "the OpenGL visualiser is not available in this build\n" );
			return 2;
		}
		else if ( a == "-o" || ( a.rfind( "-o", 0 ) == 0 && a.size() > 2 && a[ 2 ] != '-' ) )
			out = a.size() > 2 ? a.substr( 2 ) : val( "-o" );
		else if ( is( "-s", "--sample-per-pixel" ) )
			spp = unsigned( std::strtoul( ( a.size() > 2 && a[ 1 ] != '-' ? a.substr( 2 ) : val( "-s" ) ).c_str(), nullptr, 10 ) );
		else if ( a.rfind( "--resolution", 0 ) == 0 )
			res = val( "--resolution" );
		else if ( is( "-k", "--kernel" ) )
			kernel = a.size() > 2 && a[ 1 ] != '-' ? a.substr( 2 ) : val( "-k" );
		else if ( is( "-t", "--tracer" ) )
			tracer = a.size() > 2 && a[ 1 ] != '-' ? a.substr( 2 ) : val( "-t" );
		else if ( is( "-a", "--allocator" ) )
			( void )( a.size() > 2 && a[ 1 ] != '-' ? a.substr( 2 ) : val( "-a" ) );
		else if ( a.rfind( "--pfm", 0 ) == 0 )
			pfm = val( "--pfm" );
		else if ( !a.empty() && a[ 0 ] != '-' && scene.empty() )
			scene = a;
		else
		{
			std::fprintf( stderr, "unknown option %s\n", a.c_str() );
			return 2;
		}
	}
	if ( scene.empty() )
	{
		usage();
		return 2;
	}
	unsigned w = 1024, h = 768;
	if ( std::sscanf( res.c_str(), "%ux%u", &w, &h ) != 2 || !w || !h )
	{
		std::fprintf( stderr, "bad resolution %s\n", res.c_str() );
		return 2;
	}
	std::printf( "Sample %u points per pixel, %ux%u, kernel %s, tracer %s\n", spp, w, h, kernel.c_str(), tracer.c_str() );
	int rc = cr_render_file( scene.c_str(), out.c_str(), pfm.empty() ? nullptr : pfm.c_str(), spp, w, h, kernel.c_str(),
							 tracer.c_str() );
	if ( rc != CR_OK )
	{
		std::fprintf( stderr, "fatal: %s\n", cr_last_error() );
		return 1;
	}
	std::printf( "Written to '%s'\n", out.c_str() );
	return 0;
}
