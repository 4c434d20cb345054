// Json.h -- a minimal JSON document model and parser (internal), shared by the result files
// (Output.cpp) and the JSON tuning-script loader (TuningLoader.cpp).
#pragma once

#include <cctype>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace ktt::json
{

struct Json
{
    enum class Kind { Null, Bool, Number, String, Array, Object } kind = Kind::Null;
    bool boolean = false;
    double number = 0.0;
    bool integral = false;
    int64_t integer = 0;
    std::string text;
    std::vector<Json> items;
    std::vector<std::pair<std::string, Json>> members;

    const Json* Find(const std::string& key) const
    {
        for (const auto& [k, v] : members)
        {
            if (k == key)
            {
                return &v;
            }
        }

        return nullptr;
    }

    double NumberOr(const std::string& key, const double fallback) const
    {
        const Json* v = Find(key);
        return v && v->kind == Kind::Number ? v->number : fallback;
    }

    std::string StringOr(const std::string& key, const std::string& fallback) const
    {
        const Json* v = Find(key);
        return v && v->kind == Kind::String ? v->text : fallback;
    }
};

class Parser
{
public:
    explicit Parser(const std::string& text) : m_Text(text), m_Pos(0) {}

    Json Parse()
    {
        Json value = Value();
        Skip();

        if (m_Pos != m_Text.size())
        {
            throw std::runtime_error("Trailing characters in JSON document");
        }

        return value;
    }

private:
    const std::string& m_Text;
    size_t m_Pos;

    void Skip()
    {
        while (m_Pos < m_Text.size() && std::isspace(static_cast<unsigned char>(m_Text[m_Pos])))
        {
            ++m_Pos;
        }
    }

    char Peek()
    {
        Skip();

        if (m_Pos >= m_Text.size())
        {
            throw std::runtime_error("Unexpected end of JSON document");
        }

        return m_Text[m_Pos];
    }

    void Expect(const char c)
    {
        if (Peek() != c)
        {
            throw std::runtime_error(std::string("Expected '") + c + "' in JSON document");
        }

        ++m_Pos;
    }

    std::string String()
    {
        Expect('"');
        std::string out;

        while (m_Pos < m_Text.size() && m_Text[m_Pos] != '"')
        {
            char c = m_Text[m_Pos++];

            if (c == '\\' && m_Pos < m_Text.size())
            {
                const char e = m_Text[m_Pos++];

                switch (e)
                {
                case 'n': out += '\n'; break;
                case 't': out += '\t'; break;
                case 'r': out += '\r'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'u':
                {
                    const unsigned code = static_cast<unsigned>(std::stoul(m_Text.substr(m_Pos, 4), nullptr, 16));
                    m_Pos += 4;
                    out += code < 0x80 ? static_cast<char>(code) : '?';
                    break;
                }
                default: out += e; break;
                }
            }
            else
            {
                out += c;
            }
        }

        Expect('"');
        return out;
    }

    Json Value()
    {
        Json v;
        const char c = Peek();

        if (c == '{')
        {
            v.kind = Json::Kind::Object;
            ++m_Pos;

            if (Peek() == '}')
            {
                ++m_Pos;
                return v;
            }

            while (true)
            {
                std::string key = String();
                Expect(':');
                v.members.emplace_back(key, Value());

                if (Peek() == ',')
                {
                    ++m_Pos;
                    continue;
                }

                Expect('}');
                return v;
            }
        }

        if (c == '[')
        {
            v.kind = Json::Kind::Array;
            ++m_Pos;

            if (Peek() == ']')
            {
                ++m_Pos;
                return v;
            }

            while (true)
            {
                v.items.push_back(Value());

                if (Peek() == ',')
                {
                    ++m_Pos;
                    continue;
                }

                Expect(']');
                return v;
            }
        }

        if (c == '"')
        {
            v.kind = Json::Kind::String;
            v.text = String();
            return v;
        }

        if (m_Text.compare(m_Pos, 4, "true") == 0)
        {
            m_Pos += 4;
            v.kind = Json::Kind::Bool;
            v.boolean = true;
            return v;
        }

        if (m_Text.compare(m_Pos, 5, "false") == 0)
        {
            m_Pos += 5;
            v.kind = Json::Kind::Bool;
            return v;
        }

        if (m_Text.compare(m_Pos, 4, "null") == 0)
        {
            m_Pos += 4;
            return v;
        }

        const size_t start = m_Pos;

        while (m_Pos < m_Text.size() && (std::isdigit(static_cast<unsigned char>(m_Text[m_Pos])) || m_Text[m_Pos] == '-'
            || m_Text[m_Pos] == '+' || m_Text[m_Pos] == '.' || m_Text[m_Pos] == 'e' || m_Text[m_Pos] == 'E'))
        {
            ++m_Pos;
        }

        if (start == m_Pos)
        {
            throw std::runtime_error("Invalid JSON value");
        }

        const std::string token = m_Text.substr(start, m_Pos - start);
        v.kind = Json::Kind::Number;
        v.number = std::stod(token);
        v.integral = token.find_first_of(".eE") == std::string::npos;

        if (v.integral)
        {
            v.integer = std::stoll(token);
        }

        return v;
    }
};

} // namespace ktt::json
