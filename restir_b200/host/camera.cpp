// Camera and shadow-face matrices. The reference takes them from bx
// (mtxLookAt, mtxProj with Handedness::Right, camera.cpp:107-124,
// renderer.cpp:531-563), whose sources are not part of the reference; these
// are the standard right-handed forms with NDC depth in [0, 1], row-major,
// clip = M * v.
#include "bvh_build.h"

#include <algorithm>
#include <cmath>

namespace restir
{

void lookAtRH(const float* eye, const float* at, const float* up, float* out)
{
	double f[3] = { double(at[0]) - eye[0], double(at[1]) - eye[1], double(at[2]) - eye[2] };
	double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
	for (double& v : f)
	{
		v /= fl;
	}
	double s[3] = { f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0] };
	double sl = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
	for (double& v : s)
	{
		v /= sl;
	}
	double u[3] = { s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0] };
	const double m[16] = {
		s[0], s[1], s[2], -(s[0] * eye[0] + s[1] * eye[1] + s[2] * eye[2]),
		u[0], u[1], u[2], -(u[0] * eye[0] + u[1] * eye[1] + u[2] * eye[2]),
		-f[0], -f[1], -f[2], (f[0] * eye[0] + f[1] * eye[1] + f[2] * eye[2]),
		0.0, 0.0, 0.0, 1.0,
	};
	for (int i = 0; i < 16; ++i)
	{
		out[i] = float(m[i]);
	}
}

void perspectiveRH(float fovyRadians, float aspect, float nearPlane, float farPlane, float* out)
{
	const double h = 1.0 / std::tan(0.5 * double(fovyRadians));
	const double w = h / double(aspect);
	const double range = double(nearPlane) - double(farPlane);
	const double m[16] = {
		w, 0.0, 0.0, 0.0,
		0.0, h, 0.0, 0.0,
		0.0, 0.0, double(farPlane) / range, double(nearPlane) * double(farPlane) / range,
		0.0, 0.0, -1.0, 0.0,
	};
	for (int i = 0; i < 16; ++i)
	{
		out[i] = float(m[i]);
	}
}

void multiply(const float* a, const float* b, float* out)
{
	float r[16];
	for (int i = 0; i < 4; ++i)
	{
		for (int j = 0; j < 4; ++j)
		{
			double sum = 0.0;
			for (int k = 0; k < 4; ++k)
			{
				sum += double(a[i * 4 + k]) * double(b[k * 4 + j]);
			}
			r[i * 4 + j] = float(sum);
		}
	}
	for (int i = 0; i < 16; ++i)
	{
		out[i] = r[i];
	}
}

// Gauss-Jordan elimination with partial pivoting, in double precision.
bool invert(const float* m, float* out)
{
	double a[4][8];
	for (int i = 0; i < 4; ++i)
	{
		for (int j = 0; j < 4; ++j)
		{
			a[i][j] = m[i * 4 + j];
			a[i][j + 4] = i == j ? 1.0 : 0.0;
		}
	}
	for (int col = 0; col < 4; ++col)
	{
		int pivot = col;
		for (int r = col + 1; r < 4; ++r)
		{
			if (std::fabs(a[r][col]) > std::fabs(a[pivot][col]))
			{
				pivot = r;
			}
		}
		if (a[pivot][col] == 0.0)
		{
			return false;
		}
		for (int j = 0; j < 8; ++j)
		{
			std::swap(a[col][j], a[pivot][j]);
		}
		const double inv = 1.0 / a[col][col];
		for (int j = 0; j < 8; ++j)
		{
			a[col][j] *= inv;
		}
		for (int r = 0; r < 4; ++r)
		{
			if (r != col && a[r][col] != 0.0)
			{
				const double f = a[r][col];
				for (int j = 0; j < 8; ++j)
				{
					a[r][j] -= f * a[col][j];
				}
			}
		}
	}
	for (int i = 0; i < 4; ++i)
	{
		for (int j = 0; j < 4; ++j)
		{
			out[i * 4 + j] = float(a[i][j + 4]);
		}
	}
	return true;
}

} // namespace restir

extern "C" void restir_camera_matrices(const float* eye, float yaw, float pitch, float aspect, const float* center,
	float radius, float* view, float* projection)
{
	const float cp = std::cos(pitch);
	const float forward[3] = { -cp * std::sin(yaw), -std::sin(pitch), -cp * std::cos(yaw) };
	const float at[3] = { eye[0] + forward[0], eye[1] + forward[1], eye[2] + forward[2] };
	const float up[3] = { 0.0f, 1.0f, 0.0f };
	restir::lookAtRH(eye, at, up, view);
	const float d[3] = { eye[0] - center[0], eye[1] - center[1], eye[2] - center[2] };
	const float farPlane = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + 2.0f * radius;
	restir::perspectiveRH(48.0f * 3.14159265358979f / 180.0f, aspect, 0.05f * radius, std::max(farPlane, 2.5f * radius),
		projection);
}
