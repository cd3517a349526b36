// Checkpoint file with a running CRC-32, in the byte format of the
// reference's src/file.h:15-132: data, then the 32-bit seal
// (~crc) ^ 0xa23777ac over everything written before it.  CRC-32 is the
// standard reflected polynomial 0xEDB88320 (table method).
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <stdexcept>

class ckfile
{
	std::string _name;
	FILE * _f = nullptr;
	uint32_t _crc = 0;

	static const uint32_t * table()
	{
		static uint32_t t[256];
		static bool init = false;
		if (!init)
		{
			for (uint32_t i = 0; i < 256; ++i)
			{
				uint32_t r = i;
				for (int j = 0; j < 8; ++j) r = (r & 1) ? (r >> 1) ^ 0xedb88320u : (r >> 1);
				t[i] = r;
			}
			init = true;
		}
		return t;
	}

public:
	static uint32_t crc32(uint32_t crc, const void * buf, size_t len)
	{
		const uint32_t * t = table();
		const uint8_t * p = static_cast<const uint8_t *>(buf);
		crc = ~crc;
		for (size_t i = 0; i < len; ++i) crc = (crc >> 8) ^ t[(crc ^ p[i]) & 0xff];
		return ~crc;
	}

	ckfile(const std::string & name, const char * mode) : _name(name), _f(std::fopen(name.c_str(), mode)) {}
	~ckfile() { if (_f) std::fclose(_f); }
	ckfile(const ckfile &) = delete;
	ckfile & operator=(const ckfile &) = delete;

	bool exists() const { return _f != nullptr; }

	bool read(void * p, size_t n)
	{
		if (!_f) return false;
		const size_t r = std::fread(p, 1, n, _f);
		_crc = crc32(_crc, p, n);
		return r == n;
	}

	bool write(const void * p, size_t n)
	{
		if (!_f) return false;
		const size_t r = std::fwrite(p, 1, n, _f);
		_crc = crc32(_crc, p, n);
		return r == n;
	}

	bool write_seal()
	{
		const uint32_t s = ~_crc ^ 0xa23777acu;
		return write(&s, sizeof(s));
	}

	bool check_seal()
	{
		const uint32_t expect = ~_crc ^ 0xa23777acu;
		uint32_t s = 0;
		if (!read(&s, sizeof(s))) return false;
		return s == expect;
	}
};
