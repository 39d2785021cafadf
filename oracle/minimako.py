"""A small renderer for the subset of Mako used by the reference kernels.

Test infrastructure only (see ``oracle/__init__.py``).  The reference keeps
its CUDA kernels as Mako templates (e.g. dgfs1D/std/kernels/scattering/
vhs-gll.mako) rendered at run time by ``DottedTemplateLookup``
(dgfs1D/nputil.py:66-95).  Mako is not installed here, so this module
renders the constructs those templates use -- ``<%! %>`` module blocks,
``<% %>`` code blocks, ``% for/if/elif/else/endfor/endif`` control lines and
``${expr}`` substitutions -- by translating the template into a Python
function, the way Mako itself compiles templates.
"""
import re

_CTRL = re.compile(r'^\s*%\s*(for|if|elif|else|endfor|endif|while|endwhile)\b(.*)$')


def _split_expr(text, start):
    """Return the end index of a ``${...}`` expression opened at ``start``."""
    i, depth, quote = start + 2, 1, None
    while i < len(text):
        ch = text[i]
        if quote:
            if ch == '\\':
                i += 2
                continue
            if ch == quote:
                quote = None
        elif ch in '\'"':
            quote = ch
        elif ch == '{':
            depth += 1
        elif ch == '}':
            depth -= 1
            if depth == 0:
                return i
        i += 1
    raise ValueError('unterminated ${ expression')


def _text_line(line):
    """Python statements emitting one template text line."""
    parts, pos = [], 0
    while True:
        j = line.find('${', pos)
        if j < 0:
            parts.append(repr(line[pos:]))
            break
        parts.append(repr(line[pos:j]))
        k = _split_expr(line, j)
        parts.append('str(%s)' % line[j + 2:k])
        pos = k + 1
    return '__out.append(%s)' % ' + '.join(parts)


def _dedent_block(code):
    lines = code.split('\n')
    body = [l for l in lines if l.strip()]
    if not body:
        return []
    ind = min(len(l) - len(l.lstrip()) for l in body)
    return [l[ind:] for l in lines if l.strip()]


def compile_template(src):
    """Translate template source into Python source of ``render(**kw)``."""
    module, body = [], []
    indent = 1

    def emit(stmt):
        body.append('    ' * indent + stmt)

    # pull out <%! %> and <% %> blocks (they may span lines)
    tokens = re.split(r'(<%!.*?%>|<%.*?%>)', src, flags=re.S)
    pending = ''
    for tok in tokens:
        if tok.startswith('<%!'):
            module.extend(_dedent_block(tok[3:-2]))
            continue
        if tok.startswith('<%'):
            if pending:
                raise ValueError('code block inside a text line is unsupported')
            for l in _dedent_block(tok[2:-2]):
                emit(l)
            continue
        raw = tok.split('\n')
        # join lines inside an unterminated ${ ... } expression
        lines, buf = [], None
        for line in raw:
            buf = line if buf is None else buf + '\n' + line
            try:
                _text_line(buf)
            except ValueError:
                continue
            lines.append(buf)
            buf = None
        if buf is not None:
            raise ValueError('unterminated ${ expression')
        for idx, line in enumerate(lines):
            last = idx == len(lines) - 1
            m = _CTRL.match(line)
            if m:
                kw, rest = m.group(1), m.group(2).rstrip()
                if kw in ('endfor', 'endif', 'endwhile'):
                    indent -= 1
                elif kw in ('elif', 'else'):
                    indent -= 1
                    emit(kw + rest)
                    indent += 1
                else:
                    emit(kw + rest)
                    indent += 1
                continue
            if line.lstrip().startswith('##'):
                continue
            if last:
                if line:
                    emit(_text_line(line))
            else:
                emit(_text_line(line + '\n'))
    py = '\n'.join(module) + '\n\ndef render(**__kw):\n' \
        '    globals().update(__kw)\n    __out = []\n' + '\n'.join(body) + \
        '\n    return "".join(__out)\n'
    return py


def render(src, **kwargs):
    ns = {}
    exec(compile(compile_template(src), '<template>', 'exec'), ns)
    return ns['render'](**kwargs)
