// Minimal JSON reader for the reference's scene files (nlohmann/json 2.1.0 is
// what the reference uses; this is an independent, self-contained parser of
// RFC 8259 text into a small variant tree).
#pragma once
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace cr
{
struct Json
{
	enum Type
	{
		Null,
		Bool,
		Number,
		String,
		Array,
		Object
	} type = Null;
	bool b = false;
	double num = 0;
	std::string str;
	std::vector<Json> arr;
	std::vector<std::pair<std::string, Json>> obj;  // insertion order kept

	bool is_array() const { return type == Array; }
	bool is_object() const { return type == Object; }
	bool is_number() const { return type == Number; }
	bool is_string() const { return type == String; }
	size_t size() const { return type == Array ? arr.size() : type == Object ? obj.size() : 0; }
	const Json *find( const std::string &k ) const
	{
		if ( type != Object ) return nullptr;
		for ( auto &kv : obj )
			if ( kv.first == k ) return &kv.second;
		return nullptr;
	}
	const Json &at( size_t i ) const
	{
		if ( type != Array || i >= arr.size() ) throw std::runtime_error( "json: index out of range" );
		return arr[ i ];
	}
	double number_or( const std::string &k, double d ) const
	{
		auto *j = find( k );
		if ( !j ) return d;
		if ( j->type == Bool ) return j->b ? 1 : 0;
		if ( !j->is_number() ) throw std::runtime_error( "json: '" + k + "' is not a number" );
		return j->num;
	}
	std::string string_or( const std::string &k, const std::string &d ) const
	{
		auto *j = find( k );
		if ( !j ) return d;
		if ( !j->is_string() ) throw std::runtime_error( "json: '" + k + "' is not a string" );
		return j->str;
	}
	// A float3 property: [x, y, z] (as the reference's vec serialiser writes it).
	bool vec3( const std::string &k, float out[ 3 ] ) const
	{
		auto *j = find( k );
		if ( !j ) return false;
		if ( !j->is_array() || j->size() != 3 ) throw std::runtime_error( "json: '" + k + "' is not a 3-vector" );
		for ( int i = 0; i < 3; ++i )
		{
			if ( !j->arr[ i ].is_number() ) throw std::runtime_error( "json: '" + k + "' is not a 3-vector" );
			out[ i ] = float( j->arr[ i ].num );
		}
		return true;
	}
};

class JsonParser
{
public:
	explicit JsonParser( const std::string &s ) : s_( s ) {}
	Json parse()
	{
		Json j = value( 0 );
		ws();
		if ( p_ != s_.size() ) fail( "trailing characters" );
		return j;
	}

private:
	const std::string &s_;
	size_t p_ = 0;

	[[noreturn]] void fail( const char *what )
	{
		throw std::runtime_error( std::string( "json parse error at offset " ) + std::to_string( p_ ) + ": " + what );
	}
	void ws()
	{
		while ( p_ < s_.size() && ( s_[ p_ ] == ' ' || s_[ p_ ] == '\t' || s_[ p_ ] == '\n' || s_[ p_ ] == '\r' ) ) ++p_;
	}
	bool lit( const char *w )
	{
		size_t n = std::char_traits<char>::length( w );
		if ( s_.compare( p_, n, w ) == 0 )
		{
			p_ += n;
			return true;
		}
		return false;
	}
	Json value( int depth )
	{
		if ( depth > 256 ) fail( "nesting too deep" );
		ws();
		if ( p_ >= s_.size() ) fail( "unexpected end" );
		char c = s_[ p_ ];
		Json j;
		if ( c == '{' )
		{
			j.type = Json::Object;
			++p_;
			ws();
			if ( p_ < s_.size() && s_[ p_ ] == '}' )
			{
				++p_;
				return j;
			}
			for ( ;; )
			{
				ws();
				if ( p_ >= s_.size() || s_[ p_ ] != '"' ) fail( "expected key" );
				std::string k = string();
				ws();
				if ( p_ >= s_.size() || s_[ p_ ] != ':' ) fail( "expected ':'" );
				++p_;
				Json v = value( depth + 1 );
				bool replaced = false;
				for ( auto &kv : j.obj )
					if ( kv.first == k ) kv.second = std::move( v ), replaced = true;
				if ( !replaced ) j.obj.emplace_back( std::move( k ), std::move( v ) );
				ws();
				if ( p_ < s_.size() && s_[ p_ ] == ',' )
				{
					++p_;
					continue;
				}
				if ( p_ < s_.size() && s_[ p_ ] == '}' )
				{
					++p_;
					return j;
				}
				fail( "expected ',' or '}'" );
			}
		}
		if ( c == '[' )
		{
			j.type = Json::Array;
			++p_;
			ws();
			if ( p_ < s_.size() && s_[ p_ ] == ']' )
			{
				++p_;
				return j;
			}
			for ( ;; )
			{
				j.arr.push_back( value( depth + 1 ) );
				ws();
				if ( p_ < s_.size() && s_[ p_ ] == ',' )
				{
					++p_;
					continue;
				}
				if ( p_ < s_.size() && s_[ p_ ] == ']' )
				{
					++p_;
					return j;
				}
				fail( "expected ',' or ']'" );
			}
		}
		if ( c == '"' )
		{
			j.type = Json::String;
			j.str = string();
			return j;
		}
		if ( lit( "true" ) )
		{
			j.type = Json::Bool;
			j.b = true;
			return j;
		}
		if ( lit( "false" ) )
		{
			j.type = Json::Bool;
			return j;
		}
		if ( lit( "null" ) ) return j;
		if ( c == '-' || ( c >= '0' && c <= '9' ) )
		{
			const char *b = s_.c_str() + p_;
			char *e = nullptr;
			double v = std::strtod( b, &e );
			if ( e == b ) fail( "bad number" );
			p_ += size_t( e - b );
			j.type = Json::Number;
			j.num = v;
			return j;
		}
		fail( "unexpected character" );
	}
	static void put_utf8( std::string &o, unsigned cp )
	{
		if ( cp < 0x80 )
			o += char( cp );
		else if ( cp < 0x800 )
			o += char( 0xC0 | ( cp >> 6 ) ), o += char( 0x80 | ( cp & 0x3F ) );
		else if ( cp < 0x10000 )
			o += char( 0xE0 | ( cp >> 12 ) ), o += char( 0x80 | ( ( cp >> 6 ) & 0x3F ) ), o += char( 0x80 | ( cp & 0x3F ) );
		else
			o += char( 0xF0 | ( cp >> 18 ) ), o += char( 0x80 | ( ( cp >> 12 ) & 0x3F ) ),
				o += char( 0x80 | ( ( cp >> 6 ) & 0x3F ) ), o += char( 0x80 | ( cp & 0x3F ) );
	}
	std::string string()
	{
		++p_;  // opening quote
		std::string o;
		while ( p_ < s_.size() )
		{
			char c = s_[ p_++ ];
			if ( c == '"' ) return o;
			if ( c != '\\' )
			{
				o += c;
				continue;
			}
			if ( p_ >= s_.size() ) break;
			char e = s_[ p_++ ];
			switch ( e )
			{
			case '"': o += '"'; break;
			case '\\': o += '\\'; break;
			case '/': o += '/'; break;
			case 'b': o += '\b'; break;
			case 'f': o += '\f'; break;
			case 'n': o += '\n'; break;
			case 'r': o += '\r'; break;
			case 't': o += '\t'; break;
			case 'u':
			{
				if ( p_ + 4 > s_.size() ) fail( "bad escape" );
				unsigned cp = unsigned( std::stoul( s_.substr( p_, 4 ), nullptr, 16 ) );
				p_ += 4;
				if ( cp >= 0xD800 && cp < 0xDC00 && p_ + 6 <= s_.size() && s_[ p_ ] == '\\' && s_[ p_ + 1 ] == 'u' )
				{
					unsigned lo = unsigned( std::stoul( s_.substr( p_ + 2, 4 ), nullptr, 16 ) );
					p_ += 6;
					cp = 0x10000 + ( ( cp - 0xD800 ) << 10 ) + ( lo - 0xDC00 );
				}
				put_utf8( o, cp );
				break;
			}
			default: fail( "bad escape" );
			}
		}
		fail( "unterminated string" );
	}
};

inline Json parse_json( const std::string &text ) { return JsonParser( text ).parse(); }
}  // namespace cr
